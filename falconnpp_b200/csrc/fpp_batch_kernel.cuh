// fpp_batch_kernel.cuh — the fused batched query kernel k_batch_query and its
// launch selection, shared by the per-precision translation units
// (fpp_batch_f32.cu, fpp_batch_bf16.cu, fpp_batch_fp8.cu), which instantiate
// it for fhtDim 32..512 and d <= 512 and are compiled in parallel.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "fpp_batch.h"
#include "fpp_device.cuh"
#include "fpp_rows.cuh"
#include "fpp_tc_rotate.cuh"

namespace fpp {

constexpr int kBThreads = 256;
constexpr int kBWarps = kBThreads / 32;
constexpr int kBMaxList = 1024;   // L * m entries held in shared memory
constexpr int kBMaxProbes = 1024;
constexpr int kBMaxM1 = 16;
constexpr int kBigM1 = 32;        // per-layer probes of the big-list form
constexpr int kBigMaxL = 512;     // tables of the big-list form (its replay heap lives in the top region)
constexpr int kBMaxTop = 1024;    // k * shortlist multiple, and the replay heaps
constexpr int kHT = 8192;         // shared-memory hash set for the dedupe (2^13 slots)
constexpr int kGPerLane = 8;      // candidate ids per lane per gather step
constexpr uint32_t kGStep = 32 * kGPerLane;
constexpr unsigned kHTLimit = 5120;  // unique ids before switching to the L2 bitset
static_assert(kHTLimit - 1 + kBWarps * kGStep < (unsigned)kHT, "the hash set must keep an empty slot");
constexpr uint32_t kEmpty = 0xffffffffu;
constexpr int kHistBins = 2048;   // top 11 bits of the score key

struct BatchArgs {
  const float* Xc;
  int ld;
  const unsigned char* Xrows;  // rows reranked first (fp32 = Xc, else bf16/fp8 copy)
  size_t row_bytes;
  int nchunk;
  const float* Xscale;
  const uint32_t* flips;
  const uint32_t* bucket_off;
  const int32_t* ids;
  int n, d, L, D, log2D;
  uint32_t NB;
  const float* Q;
  int nq;
  const int* q_k;
  const int* q_qprobes;
  int k_uniform, qprobes_uniform;
  int k_max, qprobes_max;  // per-query values outside [1, max] are rejected
  int shortlist_mult;
  int32_t* out;
  int out_stride;
  float* out_v;
  uint32_t* bitset;
  long long nwords;
  uint32_t* uniq;
  uint32_t* score;
  long long cap;
  float* gdump;       // [groups][FHT] fallback dumps
  float* gheap_v;     // [groups][mmax] pair heaps
  int* gheap_i;
  int mmax;
  unsigned int* work;
  unsigned int* status;  // bit 0: candidate capacity overflow; bit 1: per-query k/qProbes out of range
  const uint32_t* order;  // processing order of the queries (nullable: 0, 1, ...)
  const uint32_t* tflips;  // non-null: rotate on the tensor cores when a query keeps one probe per table
  uint32_t* dump_probes;   // parity dump (nullable): [nq][qprobes_max] probed global bucket ids
  uint32_t* dump_counts;   // parity dump (nullable): [nq][2] candidates, unique candidates
  // big-list form (qProbes > 1024, L * m > 1024 or m1 > 16): per-block lists,
  // probes and gather prefixes, per-group layer lists and replay heaps, in
  // global scratch instead of shared memory
  float* glv;
  uint32_t* glb;
  long long list_cap;
  uint32_t* gprobe;
  uint32_t* gpo;
  uint32_t* gpe;
  long long probe_cap;
  float* ggv;
  int* ggc;
  float* grhv;
  int* grhi;
  // kHashExt: the per-table lists of query q at ext_lv / ext_lb + q * ext_stride
  const float* ext_lv;
  const uint32_t* ext_lb;
  long long ext_stride;
  // kHashExt with small lists: k_probe_cut's output per query
  // (q * qprobes_max + p): probed global bucket id, bucket offset,
  // inclusive prefix of the bucket sizes; pc_n[q] = the query's qProbes
  const uint32_t* pc_g;
  const uint32_t* pc_o;
  const uint32_t* pc_pe;
  const int* pc_n;
};

// Arguments of k_probe_cut (fpp_batch_ext.cu): the probe cut of the split
// hash's per-table lists, written per query.
struct ProbeCutArgs {
  const float* ext_lv;
  const uint32_t* ext_lb;
  long long ext_stride;
  const int* q_k;
  const int* q_qprobes;
  int k_uniform, qprobes_uniform, k_max, qprobes_max;
  int L;
  const uint32_t* bucket_off;
  uint32_t* pc_g;
  uint32_t* pc_o;
  uint32_t* pc_pe;
  int* pc_n;
  int stride;  // qprobes_max
};
cudaError_t probe_cut_lists(const ProbeCutArgs& a, int nq, cudaStream_t s);

__device__ __forceinline__ int ceil_sqrt_int(int m) {
  int r = 0;
  while (r * r < m) ++r;
  return r;
}

// block-wide radix selection of the `want`-th largest key among n keys
// produced by key_at(i); returns the key; counts of keys >= it in *ge.
template <typename F>
__device__ __forceinline__ uint32_t block_select(int n, unsigned want, F key_at, uint32_t* hist, uint32_t* s_pre,
                                                 uint32_t* s_rem, unsigned* s_cnt, unsigned* ge_out) {
  if (threadIdx.x == 0) {
    *s_pre = 0;
    *s_rem = want;
  }
  uint32_t mask = 0;
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    const uint32_t pre = *s_pre;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const uint32_t k = key_at(i);
      if ((k & mask) == pre) atomicAdd(&hist[(k >> shift) & 255u], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t rem = *s_rem;
      int dg = 255;
      for (; dg > 0; --dg) {
        if (hist[dg] >= rem) break;
        rem -= hist[dg];
      }
      *s_pre = pre | ((uint32_t)dg << shift);
      *s_rem = rem;
    }
    mask |= 255u << shift;
    __syncthreads();
  }
  const uint32_t t = *s_pre;
  if (threadIdx.x == 0) *s_cnt = 0;
  __syncthreads();
  unsigned ge = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) ge += key_at(i) >= t;
  atomicAdd(s_cnt, ge);
  __syncthreads();
  *ge_out = *s_cnt;
  __syncthreads();
  return t;
}

// The bin of a kHistBins-bin histogram (counts by key bits, larger bin =
// larger keys) that holds the want-th largest key, for 1 <= want <= total:
// *bin, *above = the count in bins >= it, *inbin = the count in it.  Thread t
// owns bins [kHistBins - 8(t+1), kHistBins - 8t), scanned from the top; needs
// blockDim.x * 8 == kHistBins.  Ends with a barrier.
__device__ __forceinline__ void hist_find(const uint32_t* h, unsigned want, long long* tmp, unsigned* bin,
                                          unsigned* above_out, unsigned* inbin) {
  const int tid = threadIdx.x;
  uint32_t c[8];
  uint32_t sum = 0;
  const int hi = kHistBins - 8 * tid;
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    c[b] = h[hi - 1 - b];
    sum += c[b];
  }
  long long tot;
  const long long above = block_exclusive_scan((long long)sum, tmp, &tot);
  if (above < (long long)want && above + sum >= want) {
    long long cum = above;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      if (cum + c[b] >= want && cum < (long long)want) {
        *bin = (unsigned)(hi - 1 - b);
        *above_out = (unsigned)(cum + c[b]);
        *inbin = c[b];
      }
      cum += c[b];
    }
  }
  __syncthreads();
}

// ascending bitonic sort of n (<= kBMaxTop) 64-bit keys in shared memory
__device__ __forceinline__ void block_sort_u64(unsigned long long* a, int n) {
  int N = 1;
  while (N < n) N <<= 1;
  for (int k2 = 2; k2 <= N; k2 <<= 1)
    for (int j = k2 >> 1; j > 0; j >>= 1) {
      for (int t = threadIdx.x; t < N / 2; t += blockDim.x) {
        const int blk = t / j;
        int lo, hi;
        if (j == (k2 >> 1)) {
          lo = blk * k2 + (t - blk * j);
          hi = blk * k2 + k2 - 1 - (t - blk * j);
        } else {
          lo = blk * 2 * j + (t - blk * j);
          hi = lo + j;
        }
        if (hi < n) {
          const unsigned long long x = a[lo], y = a[hi];
          if (x > y) {
            a[lo] = y;
            a[hi] = x;
          }
        }
      }
      __syncthreads();
    }
}

constexpr int kQhStride = 36;  // 32 floats + 4 of padding: segment starts 4 banks apart

// dynamic shared memory of k_batch_query (regions reused phase by phase)
template <int GROUPS>
struct BatchSmem {
  static constexpr size_t kHt = 0;                              // hash set (gather)
  static constexpr size_t kLv = kHt + 4 * kHT;                  // lists (hash, select)
  static constexpr size_t kLb = kLv + 4 * kBMaxList;
  static constexpr size_t kProbe = kLb + 4 * kBMaxList;
  static constexpr size_t kTop = kProbe + 4 * kBMaxProbes;      // sorted (key, id) of the top-k stage
  static constexpr size_t kGv = kTop + 8 * kBMaxTop;
  static constexpr size_t kGc = kGv + 4 * GROUPS * 2 * (kBMaxM1 + 1);
  static constexpr size_t kRhv = kGc + 4 * GROUPS * 2 * (kBMaxM1 + 1);
  static constexpr size_t kRhi = kRhv + 4 * GROUPS * kBMaxM1;
  static constexpr size_t kQ = kRhi + 4 * GROUPS * kBMaxM1;
  static constexpr size_t kQx = kQ + 4 * 1024;                  // query parts of the tensor-core rerank
  static constexpr size_t kQh = kQx + 2048;                     // the query for the rotations, padded
  static constexpr size_t kBytes = kQh + 4 * kQhStride * 16;
  uint32_t* ht;
  float* lv;
  uint32_t* lb;
  uint32_t* probe;
  unsigned long long* top;
  float* gv;
  int* gc;
  float* rhv;
  int* rhi;
  float* q;  // the current query, zero padded to 1024 floats
  unsigned char* qx;
  float* qh;  // segment s (32 floats) of the query at qh + s * kQhStride: the
              // lanes of a rotation group read their segments from distinct banks
  // aliases: gather prefix arrays over the lists; the score histogram over
  // both lists (2048 u32); the probe-cut replay heap in the top region; the
  // re-score arrays and the final replay heap in the hash-set region
  __device__ uint32_t* po() const { return lb; }
  __device__ uint32_t* pe() const { return reinterpret_cast<uint32_t*>(lv); }
  __device__ uint32_t* hist() const { return reinterpret_cast<uint32_t*>(lv); }
  __device__ float* phv() const { return reinterpret_cast<float*>(top); }
  __device__ int* phi() const { return reinterpret_cast<int*>(top) + 512; }
  __device__ uint32_t* sid() const { return ht; }
  __device__ uint32_t* ssc() const { return ht + 1024; }
  __device__ float* fhv() const { return reinterpret_cast<float*>(ht + 2048); }
  __device__ int* fhi() const { return reinterpret_cast<int*>(ht + 3072); }
  __device__ explicit BatchSmem(unsigned char* p)
      : ht(reinterpret_cast<uint32_t*>(p + kHt)),
        lv(reinterpret_cast<float*>(p + kLv)),
        lb(reinterpret_cast<uint32_t*>(p + kLb)),
        probe(reinterpret_cast<uint32_t*>(p + kProbe)),
        top(reinterpret_cast<unsigned long long*>(p + kTop)),
        gv(reinterpret_cast<float*>(p + kGv)),
        gc(reinterpret_cast<int*>(p + kGc)),
        rhv(reinterpret_cast<float*>(p + kRhv)),
        rhi(reinterpret_cast<int*>(p + kRhi)),
        q(reinterpret_cast<float*>(p + kQ)),
        qx(p + kQx),
        qh(reinterpret_cast<float*>(p + kQh)) {}
};

template <int FHT>
constexpr size_t batch_smem_bytes() {
  return BatchSmem<kBThreads / Geo<FHT>::G>::kBytes;
}

__device__ __forceinline__ uint32_t ht_slot(uint32_t id) { return (id * 2654435761u) >> (32 - 13); }
// the probe stride of an id (double hashing): odd, so with the power-of-two
// table every slot is reached, and from an independent multiplier, so ids
// that share a first slot take different paths (linear probing's clusters
// made a 256-id step wait for chains of ~11 probes at 55 % fill)
__device__ __forceinline__ uint32_t ht_step(uint32_t id) { return ((id * 0x85EBCA6Bu) >> (32 - 13)) | 1u; }

// The shortlist, the exact FP32 re-score and the top-k of one query
// (FalconnPP.cpp:642-706) from its U unique candidates uq[0..U) with their
// first-pass scores sc[0..U) (FP32 key bits) and the 2048-bin histogram of
// the scores' top 11 key bits in sm.hist(); the query's FP32 vector is in
// sm.q.  Writes orow / ovrow.  Every thread of the block calls it.  Returns
// whether bitset words still need clearing (use_bitset and the unique list
// kept).
struct FinishShared {
  uint32_t* hist;  // 256 bins for the radix selection
  uint32_t *s_pre, *s_rem;
  unsigned *s_cnt, *s_sel, *s_bstar, *s_above, *s_inbin;
  long long* tmp;
};

template <int MODE, int VI32, int GROUPS>
__device__ __forceinline__ bool finish_query(const BatchArgs& a, const BatchSmem<GROUPS>& sm,
                                             unsigned long long* s_top, uint32_t* uq, uint32_t* sc, unsigned U, int k,
                                             int32_t* orow, float* ovrow, bool use_bitset, uint32_t* bits,
                                             const FinishShared& fs, int tid, int warp, int lane) {
  uint32_t* s_hist = sm.hist();
  const unsigned kk = (unsigned)k;
  const unsigned R = MODE == kRowsF32 ? kk : min((unsigned)kBMaxTop, kk * (unsigned)a.shortlist_mult);
  unsigned nsel = U;
  bool exact = true;
  uint32_t* sid = sm.sid();
  uint32_t* ssc = sm.ssc();
  // the shortlist (ids and first scores) goes to sid/ssc: every candidate
  // whose key reaches the cut t, which is the bin of the R-th largest key
  // (refined by the next 11 key bits when that bin holds many)
  if (U > R) {
    hist_find(s_hist, R, fs.tmp, fs.s_bstar, fs.s_above, fs.s_inbin);
    const uint32_t bstar = *fs.s_bstar;
    const unsigned above = *fs.s_above, inbin = *fs.s_inbin;
    bool take = true;
    uint32_t t = bstar << 21;
    if (above <= (unsigned)kBMaxTop) {
      if (above > R + R / 2 + 32) {
        for (int i = tid; i < kHistBins; i += kBThreads) s_hist[i] = 0u;
        __syncthreads();
        for (unsigned i = tid; i < U; i += kBThreads) {
          const uint32_t key = ord_key_bits(sc[i]);
          if ((key >> 21) == bstar) atomicAdd(s_hist + ((key >> 10) & (kHistBins - 1)), 1u);
        }
        __syncthreads();
        hist_find(s_hist, R - (above - inbin), fs.tmp, fs.s_bstar, fs.s_above, fs.s_inbin);
        t |= *fs.s_bstar << 10;
      }
    } else {
      // very many equal top bits: radix selection of the R-th key
      unsigned ge;
      t = block_select((int)U, R, [&](int i) { return ord_key_bits(sc[i]); }, fs.hist, fs.s_pre, fs.s_rem, fs.s_cnt,
                       &ge);
      if (MODE == kRowsF32 && ge != R) {
        exact = false;
        take = false;
      }
    }
    if (take) {
      if (tid == 0) *fs.s_sel = 0;
      __syncthreads();
      for (unsigned i = tid; i < U; i += kBThreads) {
        const uint32_t key = ord_key_bits(sc[i]);
        if (key >= t) {
          const unsigned pos = atomicAdd(fs.s_sel, 1u);
          if (pos < (unsigned)kBMaxTop) {
            sid[pos] = uq[i];
            ssc[pos] = sc[i];
          }
        }
      }
      __syncthreads();
      nsel = min(*fs.s_sel, (unsigned)kBMaxTop);
    }
  } else {
    for (unsigned i = tid; i < U; i += kBThreads) {
      sid[i] = uq[i];
      ssc[i] = sc[i];
    }
    __syncthreads();
  }
  if (exact) {
    if (MODE != kRowsF32) {
      // exact FP32 re-score of the shortlist with the parity dot order
      rerank_rows<kRowsF32, VI32>(sid, nsel, ssc, sm.q, reinterpret_cast<const unsigned char*>(a.Xc),
                                  (size_t)a.ld * 4, a.ld / 4, nullptr, warp, kBWarps, lane, nullptr);
      __syncthreads();
    }
    const unsigned kept = min(nsel, kk);
    unsigned dup = 0;
    // s_top[0..kept): the best candidates by (score desc, id asc).  Equal
    // FP32 scores in the kept list, or at the k-th place, leave the order to
    // the reference's heap (dup).
    if (nsel <= 2u * kBThreads) {
      // rank by counting: no sort, two barriers
      for (unsigned i = tid; i < nsel; i += kBThreads) {
        const uint32_t ki = ord_key_bits(ssc[i]);
        const uint32_t ii = sid[i];
        unsigned gt = 0, eq = 0, before = 0;
        for (unsigned j = 0; j < nsel; ++j) {
          const uint32_t kj = ord_key_bits(ssc[j]);
          gt += kj > ki;
          eq += kj == ki;
          before += (kj == ki) & (sid[j] < ii);
        }
        const unsigned r = gt + before;
        if (r < kept) s_top[r] = ((unsigned long long)(~ki) << 32) | ii;
        dup |= (eq > 1u) & (gt < kk);
      }
    } else {
      for (unsigned i = tid; i < nsel; i += kBThreads)
        s_top[i] = ((unsigned long long)(~ord_key_bits(ssc[i])) << 32) | sid[i];
      __syncthreads();
      block_sort_u64(s_top, (int)nsel);
      for (unsigned i = tid; i + 1 < nsel && i < kk; i += kBThreads)
        dup |= (s_top[i] >> 32) == (s_top[i + 1] >> 32);
    }
    exact = !__syncthreads_or(dup);
    if (exact) {
      for (int j = tid; j < k; j += kBThreads) {
        if ((unsigned)j < kept) {
          orow[j] = (int32_t)(uint32_t)s_top[j];
          if (ovrow) ovrow[j] = __uint_as_float(ord_key_inv_dev(~(uint32_t)(s_top[j] >> 32)));
        } else {
          orow[j] = 0;
          if (ovrow) ovrow[j] = 0.0f;
        }
      }
    }
  }
  bool bits_dirty = use_bitset;
  if (!exact) {
    // the reference's min-heap over the candidates in ascending id order
    // (FalconnPP.cpp:633-673): all of them in FP32 mode, the shortlist otherwise
    const bool whole = (MODE == kRowsF32);
    const unsigned nc = whole ? U : nsel;
    uint32_t* cid = uq;
    uint32_t* csc = sc;
    if (!whole) {
      for (unsigned i = tid; i < nc; i += kBThreads) {  // the shortlist with its exact FP32 scores
        cid[i] = sid[i];
        csc[i] = ssc[i];
      }
      __syncthreads();
      if (use_bitset) {  // the unique list was overwritten: clear every word
        for (long long w = tid; w < a.nwords; w += kBThreads) bits[w] = 0u;
        bits_dirty = false;
      }
    }
    block_bitonic_sort_u32(cid, csc, (int)nc);
    if (tid == 0) {
      float* hv = sm.fhv();
      int* hi = sm.fhi();
      int n = 0;
      for (unsigned i = 0; i < nc; ++i) topp_offer<int>(hv, hi, n, k, __uint_as_float(csc[i]), (int)cid[i]);
      for (int j = n; j < k; ++j) {
        orow[j] = 0;
        if (ovrow) ovrow[j] = 0.0f;
      }
      for (int j = n - 1; j >= 0; --j) {
        orow[j] = hi[0];
        if (ovrow) ovrow[j] = hv[0];
        heap_pop<true, int>(hv, hi, n);
      }
    }
    __syncthreads();
  }
  return bits_dirty;
}

// HASH: kHashAuto rotates on the tensor cores where a query keeps one probe
// per table (and a.tflips is set), exactly otherwise; kHashTC only on the
// tensor cores (the host uses it when every query of the batch keeps one
// probe per table), which leaves the exact rotation's registers out;
// kHashExt takes every query's per-table probe lists from the exact FP32
// hash kernel launched before it (hash_lists, the plain path's k_query_hash
// with per-query qProbes), so the rotation's registers and spills leave the
// gather / rerank loop entirely.
enum HashKind : int { kHashAuto = 0, kHashTC = 1, kHashExt = 2 };

template <int FHT, int MODE, int VI, int VI32, int HASH = kHashAuto, bool BIGL = false>
__global__ void __launch_bounds__(kBThreads, MODE == kRowsF32 ? 2 : 3) k_batch_query(BatchArgs a) {
  static_assert(HASH != kHashTC || (FHT == 256 && MODE != kRowsF32), "tensor-core rotation: fhtDim 256, BF16/FP8");
  static_assert(!(BIGL && HASH == kHashTC), "the big-list form hashes in FP32");
  constexpr int M1C = BIGL ? kBigM1 : kBMaxM1;  // per-layer list capacity
  // the probe cut and the bucket ranges come from k_probe_cut
  constexpr bool PCUT = HASH == kHashExt && !BIGL;
  constexpr int E = Geo<FHT>::E;
  constexpr int G = Geo<FHT>::G;
  constexpr int WORDS = Geo<FHT>::WORDS;
  constexpr int GROUPS = kBThreads / G;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BatchSmem<GROUPS> sm(smem_raw);
  float* s_lv = BIGL ? a.glv + (size_t)blockIdx.x * a.list_cap : sm.lv;
  uint32_t* s_lb = BIGL ? a.glb + (size_t)blockIdx.x * a.list_cap : sm.lb;
  uint32_t* s_probe = BIGL ? a.gprobe + (size_t)blockIdx.x * a.probe_cap : sm.probe;
  unsigned long long* s_top = sm.top;
  __shared__ uint32_t hist[256];
  __shared__ uint32_t s_pre, s_rem;
  __shared__ unsigned s_cnt, s_u, s_sel, s_q, s_ovf, s_bstar, s_above, s_inbin, s_qmax;
  __shared__ long long tmp[32];

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int gl = lane & (G - 1);
  const int grp = tid / G;
  const unsigned gmask = (G == 32) ? kFullMask : (((1u << G) - 1u) << (lane & ~(G - 1)));
  const long long gid = (long long)blockIdx.x * GROUPS + grp;
  // the group's two per-layer lists and its replay heap
  float* grp_v = BIGL ? a.ggv + gid * 2 * (M1C + 1) : sm.gv + grp * 2 * (M1C + 1);
  int* grp_c = BIGL ? a.ggc + gid * 2 * (M1C + 1) : sm.gc + grp * 2 * (M1C + 1);
  float* grp_rhv = BIGL ? a.grhv + gid * M1C : sm.rhv + grp * M1C;
  int* grp_rhi = BIGL ? a.grhi + gid * M1C : sm.rhi + grp * M1C;
  uint32_t* bits = a.bitset + (size_t)blockIdx.x * a.nwords;
  uint32_t* uq = a.uniq + (size_t)blockIdx.x * a.cap;
  uint32_t* sc = a.score + (size_t)blockIdx.x * a.cap;
  float* ydump = a.gdump + gid * FHT;
  float* ph_v = a.gheap_v + gid * (long long)a.mmax;
  int* ph_i = a.gheap_i + gid * (long long)a.mmax;
  const int L = a.L;
  for (int i = tid; i < kHT; i += kBThreads) sm.ht[i] = kEmpty;

  for (;;) {
    __syncthreads();
    if (tid == 0) {
      s_q = atomicAdd(a.work, 1u);
      s_qmax = 0u;
    }
    __syncthreads();
    const unsigned qu = s_q;
    if (qu >= (unsigned)a.nq) break;
    const int q = a.order ? (int)a.order[qu] : (int)qu;
    const int k = a.q_k ? a.q_k[q] : a.k_uniform;
    const int Qp = a.q_qprobes ? a.q_qprobes[q] : a.qprobes_uniform;
    if (k < 1 || k > a.k_max || Qp < 1 || Qp > a.qprobes_max) {  // block-uniform
      if (tid == 0) atomicOr(a.status, 2u);
      for (int j = tid; j < a.out_stride; j += kBThreads) a.out[(size_t)q * a.out_stride + j] = -1;
      continue;
    }
    const int m = (2 * Qp + L - 1) / L;  // ceil(2.0 * qProbes / L), FalconnPP.cpp:336
    const int m1 = ceil_sqrt_int(m);     // ceil(sqrt(m)), FalconnPP.cpp:337
    const int M = L * m;
    const float* qv = a.Q + (size_t)q * a.d;
    if constexpr (HASH == kHashExt) {
      s_lv = const_cast<float*>(a.ext_lv) + (size_t)q * a.ext_stride;
      s_lb = const_cast<uint32_t*>(a.ext_lb) + (size_t)q * a.ext_stride;
    }
    {
      float amax = 0.0f;  // max |q| (the E4M3 query scale)
      for (int i = tid; i < 1024; i += kBThreads) {
        const float x = i < a.d ? qv[i] : 0.0f;
        sm.q[i] = x;
        if (HASH != kHashExt && i < G * E) sm.qh[(i >> 5) * kQhStride + (i & 31)] = x;
        amax = fmaxf(amax, fabsf(x));
      }
      if (MODE != kRowsF32) {
#pragma unroll
        for (int o = 16; o; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(kFullMask, amax, o));
        if (lane == 0) atomicMax(&s_qmax, __float_as_uint(amax));  // non-negative: bits order as values
      }
    }
    __syncthreads();

    // ---- 1. rotate + hash every table (FalconnPP.cpp:358-531)
    if (HASH != kHashExt && FHT == 256 && MODE != kRowsF32 && (HASH == kHashTC || (a.tflips && m == 1))) {
      // low-precision modes with one probe per table: each warp rotates one
      // (table, layer) at a time on the tensor cores and keeps its best
      // coordinate (ties to the smaller position)
      float scale = 1.0f;
      {
        const float qm = __uint_as_float(s_qmax);
        int ex = 0;
        if (qm > 0.0f) {
          frexpf(qm, &ex);  // qm < 2^ex
          scale = __int_as_float(min(254, max(1, 123 - ex)) << 23);  // 2^(-ex-4): max |q| * scale < 1/16
        }
      }
      const H16Frags hf(lane);
      uint32_t qb[2][2];
      tc_query_frags(sm.q, scale, lane, qb);
      // two (table, layer) items per warp at a time: item it and it + kBWarps
      // (an item past the end repeats the first, and its result is dropped)
      for (int it = warp; it < 2 * L; it += 2 * kBWarps) {
        const int it2 = it + kBWarps < 2 * L ? it + kBWarps : it;
        const uint32_t* const tw[2] = {a.tflips + ((size_t)((it & 1) * L + (it >> 1)) * 3) * 8,
                                       a.tflips + ((size_t)((it2 & 1) * L + (it2 >> 1)) * 3) * 8};
        float v[2];
        int code[2];
        tc_rotate_top1<2>(qb, tw, hf, lane, a.D, a.log2D, v, code);
        if (lane == 0) {
          sm.gv[it] = v[0];
          sm.gc[it] = code[0];
          sm.gv[it2] = v[1];
          sm.gc[it2] = code[1];
        }
      }
      __syncthreads();
      for (int l = tid; l < L; l += kBThreads) {
        s_lv[l] = __fadd_rn(sm.gv[2 * l], sm.gv[2 * l + 1]);
        s_lb[l] = (uint32_t)l * a.NB + (uint32_t)(sm.gc[2 * l] * 2 * a.D + sm.gc[2 * l + 1]);
      }
    } else if constexpr (HASH == kHashAuto) {
      const float* xs = sm.qh + gl * kQhStride;  // the query segment of this lane, zero padded past d
      const int cnt = min(m1 + 1, a.D);
      const int rounds = (L + GROUPS - 1) / GROUPS;
      constexpr int kGroupsPerWarp = 32 / G;
      for (int rd = 0; rd < rounds; ++rd) {
        // a warp whose groups all have no table left stops (warp-uniform)
        if (rd * GROUPS + warp * kGroupsPerWarp >= L) break;
        const int l = rd * GROUPS + grp;
        const bool active = l < L;
        const int lt = active ? l : 0;
#pragma unroll 1
        for (int layer = 0; layer < 2; ++layer) {
          float y[E];
#pragma unroll
          for (int e = 0; e < E; ++e) y[e] = xs[e];
          hd3_rotate<FHT>(y, a.flips + ((size_t)(layer * L + lt) * 3) * WORDS, gl);
          float* lv = grp_v + layer * (M1C + 1);
          int* lc = grp_c + layer * (M1C + 1);
          const bool ok = group_top_cp_checked<FHT>(y, gl, a.D, a.log2D, m1, cnt, lv, lc);
          if (!ok) {
#pragma unroll
            for (int e = 0; e < E; ++e) ydump[gl * E + e] = y[e];
            __syncwarp(gmask);
            if (gl == 0) replay_layer_topp(ydump, a.D, a.log2D, m1, grp_rhv, grp_rhi, lv, lc);
            __syncwarp(gmask);
          }
        }
        if (gl == 0 && active) {
          const float* lv1 = grp_v;
          const int* lc1 = grp_c;
          const float* lv2 = grp_v + (M1C + 1);
          const int* lc2 = grp_c + (M1C + 1);
          const uint32_t tbase = (uint32_t)l * a.NB;
          const int twoD = 2 * a.D;
          if (m == 1) {
            s_lv[l] = __fadd_rn(lv1[0], lv2[0]);
            s_lb[l] = tbase + (uint32_t)(lc1[0] * twoD + lc2[0]);
          } else {
            int hn = 0;
            for (int i = 0; i < m1; ++i)
              for (int j = 0; j < m1; ++j)
                topp_offer<int>(ph_v, ph_i, hn, m, __fadd_rn(lv1[i], lv2[j]), lc1[i] * twoD + lc2[j]);
            for (int j = m - 1; j >= 0; --j) {
              s_lv[l * m + j] = ph_v[0];
              s_lb[l * m + j] = tbase + (uint32_t)ph_i[0];
              heap_pop<true, int>(ph_v, ph_i, hn);
            }
          }
        }
        __syncwarp();
      }
    }
    __syncthreads();

    // ---- 2. global top-qProbes of the L*m lists (FalconnPP.cpp:540-582):
    // rank by counting (big lists: radix selection of the qProbes-th largest
    // score); a tie straddling the cut replays the reference's heap
    if constexpr (PCUT) {
      // k_probe_cut ranked this query's lists
    } else if constexpr (BIGL) {
      bool tie = false;
      uint32_t t = 0;
      if (Qp < M) {
        unsigned ge;
        t = block_select(M, (unsigned)Qp, [&](int i) { return ord_key(s_lv[i]); }, hist, &s_pre, &s_rem, &s_cnt, &ge);
        tie = ge != (unsigned)Qp;
      }
      if (!tie) {
        long long run = 0;
        for (int base = 0; base < M; base += kBThreads) {
          const int i = base + tid;
          const bool take = i < M && (Qp >= M || ord_key(s_lv[i]) >= t);
          long long tot;
          const long long pos = block_exclusive_scan(take ? 1 : 0, tmp, &tot) + run;
          if (take) s_probe[pos] = s_lb[i];
          run += tot;
        }
      } else if (tid == 0) {
        float* hv = sm.phv();
        int* hi = sm.phi();
        int* track = hi + L;
        int n = 0;
        for (int l = 0; l < L; ++l) {
          heap_push<false, int>(hv, hi, n, s_lv[l * m], l * m);
          track[l] = 0;
        }
        for (int pc = 0; pc < Qp; ++pc) {
          const int pos = hi[0];
          heap_pop<false, int>(hv, hi, n);
          s_probe[pc] = s_lb[pos];
          const int tb = pos / m;
          track[tb]++;
          if (track[tb] < m) heap_push<false, int>(hv, hi, n, s_lv[tb * m + track[tb]], tb * m + track[tb]);
        }
      }
      __syncthreads();
    } else {
      // the order keys of the scores, once, in the top-k region (free until
      // the replay below, which runs after the counting), padded with key 0
      // to a multiple of 4 (scores are >= 0, so their keys exceed 0)
      uint32_t* s_key = reinterpret_cast<uint32_t*>(s_top);
      const int M4 = (M + 3) >> 2;
      for (int i = tid; i < 4 * M4; i += kBThreads) s_key[i] = i < M ? ord_key(s_lv[i]) : 0u;
      __syncthreads();
      long long run = 0;
      bool tie = false;
      for (int base = 0; base < M; base += kBThreads) {
        const int i = base + tid;
        bool take = false;
        if (i < M) {
          const uint32_t ki = s_key[i];
          int gt = 0, eq = 0;
          for (int j = 0; j < M4; ++j) {
            const uint4 k4 = reinterpret_cast<const uint4*>(s_key)[j];
            gt += (k4.x > ki) + (k4.y > ki) + (k4.z > ki) + (k4.w > ki);
            eq += (k4.x == ki) + (k4.y == ki) + (k4.z == ki) + (k4.w == ki);
          }
          take = gt < Qp;
          tie |= take && gt + eq > Qp;
        }
        long long tot;
        const long long pos = block_exclusive_scan(take ? 1 : 0, tmp, &tot) + run;
        if (take && pos < Qp) s_probe[pos] = s_lb[i];
        run += tot;
      }
      if (__syncthreads_or(tie) && tid == 0) {
        float* hv = sm.phv();
        int* hi = sm.phi();
        int* track = hi + L;
        int n = 0;
        for (int l = 0; l < L; ++l) {
          heap_push<false, int>(hv, hi, n, s_lv[l * m], l * m);
          track[l] = 0;
        }
        for (int pc = 0; pc < Qp; ++pc) {
          const int pos = hi[0];
          heap_pop<false, int>(hv, hi, n);
          s_probe[pc] = s_lb[pos];
          const int tb = pos / m;
          track[tb]++;
          if (track[tb] < m) heap_push<false, int>(hv, hi, n, s_lv[tb * m + track[tb]], tb * m + track[tb]);
        }
      }
      __syncthreads();
    }
    if (!PCUT && a.dump_probes)
      for (int j = tid; j < Qp; j += kBThreads) a.dump_probes[(size_t)q * a.qprobes_max + j] = s_probe[j];

    // ---- 3. gather + dedupe (FalconnPP.cpp:584-606): the candidates of all
    // probes flattened over the warps; dedupe in a shared-memory hash set, or
    // (when a query has too many unique ids) in the block's L2 bitset
    uint32_t* s_po = BIGL ? a.gpo + (size_t)blockIdx.x * a.probe_cap : sm.po();
    uint32_t* s_pe = BIGL ? a.gpe + (size_t)blockIdx.x * a.probe_cap : sm.pe();
    if constexpr (PCUT) {
      // the ranges of the slot's probes, and their ids on the way to L2
      const size_t pb = (size_t)q * a.qprobes_max;
      for (int p = tid; p < Qp; p += kBThreads) {
        const uint32_t pe = a.pc_pe[pb + p];
        const uint32_t ex = p ? a.pc_pe[pb + p - 1] : 0u;
        const uint32_t o = a.pc_o[pb + p];
        s_pe[p] = pe;
        s_po[p] = o - ex;
        if (a.dump_probes) a.dump_probes[(size_t)q * a.qprobes_max + p] = a.pc_g[pb + p];
        const uint32_t w0 = o & ~3u, w1 = min(o + (pe - ex), w0 + 4096u) & ~3u;
        if (w1 > w0) prefetch_l2(a.ids + w0, (w1 - w0) * 4u);
      }
    } else {
      long long run = 0;
      for (int base = 0; base < Qp; base += kBThreads) {
        const int p = base + tid;
        uint32_t o = 0, sz = 0;
        if (p < Qp) {
          const uint32_t g = s_probe[p];
          o = a.bucket_off[g];
          sz = a.bucket_off[g + 1] - o;
          // the bucket's ids (the 16-byte aligned part, at most 16 KB) into L2
          const uint32_t w0 = o & ~3u, w1 = min(o + sz, w0 + 4096u) & ~3u;
          if (w1 > w0) prefetch_l2(a.ids + w0, (w1 - w0) * 4u);
        }
        long long tot;
        const long long ex = block_exclusive_scan((long long)sz, tmp, &tot) + run;
        if (p < Qp) {
          s_po[p] = o - (uint32_t)ex;  // candidate i of probe p is ids[i + s_po[p]] (mod 2^32)
          s_pe[p] = (uint32_t)(ex + sz);
        }
        run += tot;
      }
    }
    if (tid == 0) {
      s_u = 0;
      s_ovf = 0;
    }
    __syncthreads();
    const uint32_t C = s_pe[Qp - 1];
    const unsigned cap = (unsigned)a.cap;
    bool use_bitset = false;
    for (int pass = 0; pass < 2; ++pass) {
      const uint32_t per = (((C + kBWarps - 1) / kBWarps) + (kGStep - 1)) & ~(kGStep - 1);
      const uint32_t c_begin = min(C, (uint32_t)warp * per);
      const uint32_t c_end = min(C, c_begin + per);
      // the probe of the lane's next candidate, the end of that probe's
      // candidates and its id offset, kept in registers: a lane's candidate
      // positions only rise, so it advances past a probe boundary (one
      // shared-memory read) only where its candidates cross one
      int lp = 0;
      {
        int lo = 0, hi = Qp - 1;
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (s_pe[mid] > c_begin) hi = mid; else lo = mid + 1;
        }
        lp = lo;
      }
      uint32_t lend = s_pe[lp], loff = s_po[lp];
      // ids of the next step are loaded while this step is inserted
      uint32_t nxt_id[kGPerLane];
      auto load_ids = [&](uint32_t c0, uint32_t (&dst)[kGPerLane]) {
#pragma unroll
        for (int h = 0; h < kGPerLane; ++h) {
          const uint32_t i = c0 + h * 32 + lane;
          dst[h] = kEmpty;
          if (i < c_end) {
            while (i >= lend) {  // ends when i < C = s_pe[Qp - 1]
              ++lp;
              lend = s_pe[lp];
              loff = s_po[lp];
            }
            dst[h] = (uint32_t)__ldg(a.ids + (i + loff));
          }
        }
      };
      if (c_begin < c_end) load_ids(c_begin, nxt_id);
      // the hash set's fill as this warp last saw it: the total that its own
      // position reservation returned (no extra shared-memory reads per step)
      bool full = false;
      for (uint32_t c0 = c_begin; c0 < c_end; c0 += kGStep) {
        if (full) break;
        uint32_t idv[kGPerLane];
#pragma unroll
        for (int h = 0; h < kGPerLane; ++h) idv[h] = nxt_id[h];
        if (c0 + kGStep < c_end) load_ids(c0 + kGStep, nxt_id);
        bool fresh[kGPerLane];
        if (use_bitset) {
#pragma unroll
          for (int h = 0; h < kGPerLane; ++h) {
            const uint32_t id = idv[h];
            const uint32_t bit = 1u << (id & 31u);
            fresh[h] = id != kEmpty && (atomicOr(bits + (id >> 5), bit) & bit) == 0u;
          }
        } else {
          // open addressing (double hashing) in rounds: every id of the step issues its probe
          // of the round before any result is examined, so the lane waits
          // for the longest chain rather than for the sum of its chains.  At
          // most kHTLimit - 1 + kBWarps * kGStep ids are ever in the table
          // (a warp inserts at most one step after its reservation shows the
          // count at the limit; a warp with no new ids adds nothing), so an
          // empty slot always exists.
          uint32_t slot[kGPerLane], old[kGPerLane];
          bool pend = false;
#pragma unroll
          for (int h = 0; h < kGPerLane; ++h) {
            slot[h] = ht_slot(idv[h]);
            old[h] = idv[h] != kEmpty ? atomicCAS(sm.ht + slot[h], kEmpty, idv[h]) : kEmpty;  // no id: done
          }
#pragma unroll
          for (int h = 0; h < kGPerLane; ++h) pend |= old[h] != kEmpty && old[h] != idv[h];
          while (pend) {
            pend = false;
#pragma unroll
            for (int h = 0; h < kGPerLane; ++h) {
              if (old[h] != kEmpty && old[h] != idv[h]) {
                slot[h] = (slot[h] + ht_step(idv[h])) & (kHT - 1);
                old[h] = atomicCAS(sm.ht + slot[h], kEmpty, idv[h]);
              }
            }
#pragma unroll
            for (int h = 0; h < kGPerLane; ++h) pend |= old[h] != kEmpty && old[h] != idv[h];
          }
#pragma unroll
          for (int h = 0; h < kGPerLane; ++h) fresh[h] = idv[h] != kEmpty && old[h] == kEmpty;
        }
        // one position reservation per warp step
        unsigned bal[kGPerLane];
        unsigned nfresh = 0;
#pragma unroll
        for (int h = 0; h < kGPerLane; ++h) {
          bal[h] = __ballot_sync(kFullMask, fresh[h]);
          nfresh += __popc(bal[h]);
        }
        if (nfresh) {
          unsigned base = 0;
          if (lane == 0) base = atomicAdd(&s_u, nfresh);
          base = __shfl_sync(kFullMask, base, 0);
          // the warp whose reservation reaches the limit raises the flag; a
          // warp stops after the step in which its reservation shows the
          // limit reached, so it inserts at most one step past it
          if (!use_bitset && base + nfresh >= kHTLimit) {
            full = true;
            if (lane == 0) s_ovf = 1u;
          }
          const unsigned below = (1u << lane) - 1u;
#pragma unroll
          for (int h = 0; h < kGPerLane; ++h) {
            const unsigned pos = base + __popc(bal[h] & below);
            if (fresh[h] && pos < cap) uq[pos] = idv[h];
            base += __popc(bal[h]);
          }
        }
      }
      __syncthreads();
      if (use_bitset || !s_ovf) break;
      // too many unique ids for the hash set: start over with the bitset
      for (int i = tid; i < kHT; i += kBThreads) sm.ht[i] = kEmpty;
      if (tid == 0) s_u = 0;
      use_bitset = true;
      __syncthreads();
    }
    const unsigned U = s_u;
    if (a.dump_counts && tid == 0) {
      a.dump_counts[2 * (size_t)q] = C;
      a.dump_counts[2 * (size_t)q + 1] = U;
    }
    int32_t* orow = a.out + (size_t)q * a.out_stride;
    float* ovrow = a.out_v ? a.out_v + (size_t)q * a.out_stride : nullptr;
    if (U > cap) {
      if (tid == 0) atomicOr(a.status, 1u);
      for (int j = tid; j < k; j += kBThreads) {
        orow[j] = -1;
        if (ovrow) ovrow[j] = 0.0f;
      }
      for (long long w = tid; w < a.nwords; w += kBThreads) bits[w] = 0u;
      for (int i = tid; i < kHT; i += kBThreads) sm.ht[i] = kEmpty;
      continue;
    }

    // ---- 4. rerank the unique rows (FalconnPP.cpp:642-660), with a
    // histogram of the scores' top 11 key bits for the selection below
    uint32_t* s_hist = sm.hist();
    float qscale = 1.0f;
    if (MODE == kRowsFP8) {
      const float qm = __uint_as_float(s_qmax);
      qscale = qm > 0.0f ? qm / 448.0f : 1.0f;  // 448: largest finite E4M3
    }
    if (MODE != kRowsF32) fill_query_parts<MODE>(sm.q, qscale, sm.qx);
    for (int i = tid; i < kHistBins; i += kBThreads) s_hist[i] = 0u;
    __syncthreads();
    if (MODE == kRowsF32) {
      rerank_rows<MODE, VI, 2>(uq, U, sc, sm.q, a.Xrows, a.row_bytes, a.nchunk, nullptr, warp, kBWarps, lane,
                               s_hist);
    } else if (a.nchunk <= 16 && 9 * 16 * a.row_bytes <= (size_t)(4 * kHT) &&
               7 * 16 * a.row_bytes <= BatchSmem<GROUPS>::kQ - BatchSmem<GROUPS>::kProbe) {
      // two tiles in flight per warp, both staged in shared memory that the
      // rerank leaves idle: the hash-set region (reset at the end of the
      // query) holds every warp's first stage and warp 7's second, the
      // probe list, top-k and rotation regions (unused until the shortlist)
      // the second stages of warps 0..6
      const size_t sb = 16 * a.row_bytes;
      unsigned char* st0 = smem_raw + (size_t)warp * sb;
      unsigned char* st1 = warp < kBWarps - 1 ? smem_raw + BatchSmem<GROUPS>::kProbe + (size_t)warp * sb
                                              : smem_raw + (size_t)kBWarps * sb;
      rerank_rows_mma_2stage<MODE>(uq, U, sc, sm.qx, a.Xrows, a.row_bytes, a.nchunk, a.Xscale, qscale, warp,
                                   kBWarps, lane, s_hist, st0, st1);
    } else {
      rerank_rows_mma<MODE>(uq, U, sc, sm.qx, a.Xrows, a.row_bytes, a.nchunk, a.Xscale, qscale, warp, kBWarps,
                            lane, s_hist);
    }
    __syncthreads();

    // ---- 5. shortlist by the first scores, exact FP32 re-score, top-k
    const FinishShared fs{hist, &s_pre, &s_rem, &s_cnt, &s_sel, &s_bstar, &s_above, &s_inbin, tmp};
    const bool bits_dirty =
        finish_query<MODE, VI32, GROUPS>(a, sm, s_top, uq, sc, U, k, orow, ovrow, use_bitset, bits, fs, tid, warp, lane);
    // ---- 6. leave the hash set empty and the bitset clear
    {
      const uint4 e4 = make_uint4(kEmpty, kEmpty, kEmpty, kEmpty);
      uint4* h4 = reinterpret_cast<uint4*>(sm.ht);
      for (int i = tid; i < kHT / 4; i += kBThreads) h4[i] = e4;
    }
    if (bits_dirty)
      for (unsigned i = tid; i < U; i += kBThreads) bits[uq[i] >> 5] = 0u;
  }
}


struct KernelSel {
  const void* fn;
  size_t smem;
};

template <int FHT, int MODE, int VI, int VI32, int HASH = kHashAuto, bool BIGL = false>
static KernelSel kernel_ptr() {
  const void* fn = reinterpret_cast<const void*>(&k_batch_query<FHT, MODE, VI, VI32, HASH, BIGL>);
  const size_t smem = batch_smem_bytes<FHT>();
  cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  return KernelSel{fn, smem};
}

template <int MODE, int VI, int VI32, bool BIGL = false>
static KernelSel pick_fht(int fht) {
  switch (fht) {
    case 32: return kernel_ptr<32, MODE, VI, VI32, kHashAuto, BIGL>();
    case 64: return kernel_ptr<64, MODE, VI, VI32, kHashAuto, BIGL>();
    case 128: return kernel_ptr<128, MODE, VI, VI32, kHashAuto, BIGL>();
    case 256: return kernel_ptr<256, MODE, VI, VI32, kHashAuto, BIGL>();
    case 512: return kernel_ptr<512, MODE, VI, VI32, kHashAuto, BIGL>();
    default: return KernelSel{nullptr, 0};
  }
}

// per-precision selection (VI: 16-byte chunks per virtual lane of the FP32
// first rerank; VI32: of the FP32 re-score), defined in fpp_batch_{f32,bf16,fp8}.cu
KernelSel pick_kernel_f32(int fht, int d);
KernelSel pick_kernel_bf16(int fht, int d, bool tc_only);
KernelSel pick_kernel_fp8(int fht, int d, bool tc_only);
KernelSel pick_kernel_big(int fht, int mode, int d);  // fpp_batch_big.cu
KernelSel pick_kernel_ext(int mode, int d, bool big);  // fpp_batch_ext.cu

inline int vi_of(int d, int epc) {
  const int v = ((d + epc - 1) / epc + 31) / 32;
  return v <= 1 ? 1 : v <= 2 ? 2 : 4;
}

}  // namespace fpp
