// fpp_build.cu — index construction on the GPU (FalconnPP::build2Layers_1D,
// src/FalconnPP.cpp:21-303), re-designed for B200:
//
//   1. centring: per-dimension chunked FP32 sums -> mean -> x - mean, stored
//      point-major in HBM (FalconnPP.cpp:33-34);
//   2. k_build_hash: one group of FHT/32 lanes per point holds the point in
//      registers and, for every table of the chunk, runs 2 layers x 3 x
//      (sign flip + shuffle FWHT), picks the top-iProbes cross-polytope codes
//      per layer and combines the two layers (FalconnPP.cpp:75-201).  Each
//      (table, point) emits iProbes (bucket, score, id) entries;
//   3. a stable LSD radix sort of the entries by (global bucket, score desc)
//      replaces the per-bucket max-heaps: entries arrive in ascending id
//      order, so equal scores stay in ascending id order;
//   4. per-bucket limits iLimit = ceil(alpha * B / iProbes) (FP32), raised to
//      min(bucket_minSize, B) (FalconnPP.cpp:233-242), give CSR offsets; the
//      first iLimit ids of every bucket are compacted into the 1D table;
//   5. where equal scores make the reference's heap order differ from
//      (score desc, id asc) — ties at the iLimit cut, and (by default) ties
//      inside the kept prefix — k_repair replays the reference's max-heap on
//      that bucket's entries and rewrites its ids in the reference's order.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>

#include <algorithm>
#include <chrono>
#include <vector>

#include "fpp_device.cuh"
#include "fpp_index.h"

namespace fpp {

#define FPP_CUDA(call)                                                                          \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) {                                                                    \
      err.code = (e_ == cudaErrorMemoryAllocation) ? kErrOutOfMemory : kErrCuda;                \
      err.msg = std::string(#call) + ": " + cudaGetErrorString(e_);                            \
      goto fail;                                                                                \
    }                                                                                           \
  } while (0)

constexpr int kCenterChunk = 1024;  // points per partial sum (the oracle uses the same)
constexpr int kMaxIProbes = 32;

int derived_fht_dim(int n_features, int n_proj) {
  // src/FalconnPP.h:96-99
  if (n_proj < n_features) return 1 << int(ceil(log2((double)n_features)));
  return 1 << int(ceil(log2((double)n_proj)));
}

// ---------------------------------------------------------------- centring
__global__ void k_center_partial(const float* __restrict__ X, long long n, int d, float* __restrict__ part) {
  const int j = blockIdx.y * blockDim.x + threadIdx.x;
  const long long c = blockIdx.x;
  if (j >= d) return;
  const long long i0 = c * kCenterChunk;
  const long long i1 = min(n, i0 + kCenterChunk);
  float s = 0.0f;
  for (long long i = i0; i < i1; ++i) s = __fadd_rn(s, X[i * d + j]);
  part[c * d + j] = s;
}

__global__ void k_center_final(const float* __restrict__ part, long long nchunks, long long n, int d,
                               float* __restrict__ mean) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= d) return;
  float s = 0.0f;
  for (long long c = 0; c < nchunks; ++c) s = __fadd_rn(s, part[c * d + j]);
  mean[j] = __fdiv_rn(s, (float)n);
}

__global__ void k_center_apply(const float* __restrict__ X, long long n, int d, int ld,
                               const float* __restrict__ mean, float* __restrict__ Xc, int* __restrict__ bad) {
  const long long total = n * (long long)ld;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long i = t / ld;
    const int j = (int)(t - i * ld);
    float v = 0.0f;
    if (j < d) {
      const float x = X[i * d + j];
      if (!isfinite(x)) atomicOr(bad, 1);
      v = __fsub_rn(x, mean[j]);
    }
    Xc[t] = v;
  }
}

// ---------------------------------------------------------------- hashing
struct HashArgs {
  const float* Xc;
  int ld, n, d;
  const uint32_t* flips;  // [2][L][3][WORDS]
  int L, l0, l1;
  int D, log2D, P;
  uint32_t NB;
  uint64_t* keys;
  uint32_t* vals;
  uint32_t* counts;  // [L * NB]
  int32_t* dump_codes;
  float* dump_scores;
};

template <int FHT>
struct HashSmem {
  static constexpr int G = Geo<FHT>::G;
  static constexpr int GROUPS = 128 / G;
  // per group: dump of one rotated vector, two top lists, one heap
  static constexpr size_t per_group = FHT * 4 + 2 * (kMaxIProbes + 1) * 8 + kMaxIProbes * 8;
  static constexpr size_t bytes = GROUPS * per_group;
};

// Block = 128 threads; a group of G lanes per point; grid-stride over points.
template <int FHT>
__global__ void __launch_bounds__(128, 4) k_build_hash(HashArgs a) {
  constexpr int E = Geo<FHT>::E;
  constexpr int G = Geo<FHT>::G;
  constexpr int WORDS = Geo<FHT>::WORDS;
  constexpr int GROUPS = HashSmem<FHT>::GROUPS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int gl = lane & (G - 1);
  const int grp = threadIdx.x / G;
  const unsigned gmask = (G == 32) ? kFullMask : (((1u << G) - 1u) << (lane & ~(G - 1)));
  unsigned char* gs = smem_raw + grp * HashSmem<FHT>::per_group;
  float* ydump = reinterpret_cast<float*>(gs);
  float* lv1 = reinterpret_cast<float*>(gs + FHT * 4);
  int* lc1 = reinterpret_cast<int*>(lv1 + (kMaxIProbes + 1));
  float* lv2 = reinterpret_cast<float*>(lc1 + (kMaxIProbes + 1));
  int* lc2 = reinterpret_cast<int*>(lv2 + (kMaxIProbes + 1));
  float* hv = reinterpret_cast<float*>(lc2 + (kMaxIProbes + 1));
  int* hi = reinterpret_cast<int*>(hv + kMaxIProbes);

  const int P = a.P;
  const int cnt = min(P + 1, a.D);
  const long long groups_total = (long long)gridDim.x * GROUPS;
  const long long n_iter = (a.n + groups_total - 1) / groups_total;
  for (long long it = 0; it < n_iter; ++it) {
    const long long pt_ll = it * groups_total + (long long)blockIdx.x * GROUPS + grp;
    const bool active = pt_ll < a.n;  // inactive groups still join every shuffle
    const int pt = active ? (int)pt_ll : 0;
    float xr[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int idx = gl * E + e;
      xr[e] = (active && idx < a.d) ? __ldg(a.Xc + (size_t)pt * a.ld + idx) : 0.0f;
    }
    for (int l = a.l0; l < a.l1; ++l) {
#pragma unroll 1
      for (int layer = 0; layer < 2; ++layer) {
        float y[E];
#pragma unroll
        for (int e = 0; e < E; ++e) y[e] = xr[e];
        hd3_rotate<FHT>(y, a.flips + ((size_t)(layer * a.L + l) * 3) * WORDS, gl);
        float* lv = layer == 0 ? lv1 : lv2;
        int* lc = layer == 0 ? lc1 : lc2;
        const bool ok = group_top_cp_checked<FHT>(y, gl, a.D, a.log2D, P, cnt, lv, lc);
        if (!ok) {  // group-uniform: replay the reference's heap scan
#pragma unroll
          for (int e = 0; e < E; ++e) ydump[gl * E + e] = y[e];
          __syncwarp(gmask);
          if (gl == 0) replay_layer_topp(ydump, a.D, a.log2D, P, hv, hi, lv, lc);
          __syncwarp(gmask);
        }
      }
      if (gl == 0 && active) {
        // two-layer combination, FalconnPP.cpp:162-189 (always replayed: P^2 offers)
        int hn = 0;
        const int twoD = 2 * a.D;
        for (int i = 0; i < P; ++i)
          for (int j = 0; j < P; ++j)
            topp_offer<int>(hv, hi, hn, P, __fadd_rn(lv2[j], lv1[i]), lc1[i] * twoD + lc2[j]);
        const size_t ebase = ((size_t)(l - a.l0) * a.n + pt) * P;
        const size_t dbase = ((size_t)l * a.n + pt) * P;
        for (int j = 0; j < P; ++j) {  // drain order of the min-heap (FalconnPP.cpp:196-201)
          const float s = hv[0];
          const int b = hi[0];
          heap_pop<true, int>(hv, hi, hn);
          a.keys[ebase + j] = ((uint64_t)((uint32_t)(l - a.l0) * a.NB + (uint32_t)b) << 32) | (uint64_t)(~ord_key(s));
          a.vals[ebase + j] = (uint32_t)pt;
          atomicAdd(a.counts + (size_t)l * a.NB + b, 1u);
          if (a.dump_codes) {
            a.dump_codes[dbase + j] = b;
            a.dump_scores[dbase + j] = s;
          }
        }
      }
      __syncwarp();
    }
  }
}

// ---------------------------------------------------------------- bucket limits
__device__ __forceinline__ uint32_t kept_of(uint32_t B, float alpha, int P, int minSize, bool* limited) {
  if (B == 0) {
    *limited = false;
    return 0;
  }
  // (int)ceil(bucket_scale * B / iProbes) in float, FalconnPP.cpp:233
  const float f = __fdiv_rn(__fmul_rn(alpha, (float)B), (float)P);
  long long lim = (long long)ceilf(f);
  *limited = false;
  if (lim < minSize) {  // FalconnPP.cpp:238-242
    lim = min((long long)minSize, (long long)B);
    *limited = true;
  }
  if (lim > (long long)B) lim = B;  // the reference would read past the bucket here
  return (uint32_t)(uint16_t)lim;   // only (uint16_t)iLimit ids are read back (FalconnPP.cpp:253, :565)
}

struct ScanArgs {
  const uint32_t* counts;  // chunk slice
  long long nb;            // buckets in the chunk
  float alpha;
  int P, minSize;
  uint32_t* segstart;      // exclusive scan of counts (chunk-local)
  uint32_t* off;           // base + exclusive scan of kept (global CSR offsets)
  unsigned long long* blk_cnt;
  unsigned long long* blk_kept;
  unsigned long long* base;   // in: ids before this chunk; out: after
  unsigned int* max_kept;
  unsigned long long* n_limited;
};

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(ScanArgs a) {
  __shared__ long long tmp[32];
  const long long t0 = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
  long long sc = 0, sk = 0, lim = 0;
  unsigned mk = 0;
  for (int i = 0; i < kScanItems; ++i) {
    const long long g = t0 + i;
    if (g < a.nb) {
      bool limited;
      const uint32_t B = a.counts[g];
      const uint32_t k = kept_of(B, a.alpha, a.P, a.minSize, &limited);
      sc += B;
      sk += k;
      lim += limited;
      mk = max(mk, k);
    }
  }
  long long tc, tk;
  block_exclusive_scan(sc, tmp, &tc);
  block_exclusive_scan(sk, tmp, &tk);
  long long tl;
  block_exclusive_scan(lim, tmp, &tl);
  if (threadIdx.x == 0) {
    a.blk_cnt[blockIdx.x] = tc;
    a.blk_kept[blockIdx.x] = tk;
    atomicAdd(a.n_limited, (unsigned long long)tl);
  }
  if (mk) atomicMax(a.max_kept, mk);
}

// single block: exclusive scan of the block sums, adds the running base
__global__ void __launch_bounds__(kScanThreads) k_scan_blocks(ScanArgs a, long long nblk) {
  __shared__ long long tmp[32];
  __shared__ long long carry_c, carry_k;
  if (threadIdx.x == 0) {
    carry_c = 0;
    carry_k = (long long)*a.base;
  }
  __syncthreads();
  for (long long s = 0; s < nblk; s += kScanThreads) {
    const long long i = s + threadIdx.x;
    const long long vc = i < nblk ? (long long)a.blk_cnt[i] : 0;
    const long long vk = i < nblk ? (long long)a.blk_kept[i] : 0;
    long long tc, tk;
    const long long ec = block_exclusive_scan(vc, tmp, &tc);
    const long long ek = block_exclusive_scan(vk, tmp, &tk);
    if (i < nblk) {
      a.blk_cnt[i] = carry_c + ec;
      a.blk_kept[i] = carry_k + ek;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      carry_c += tc;
      carry_k += tk;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *a.base = (unsigned long long)carry_k;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_down(ScanArgs a) {
  __shared__ long long tmp[32];
  const long long t0 = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
  uint32_t B[kScanItems], K[kScanItems];
  long long sc = 0, sk = 0;
  for (int i = 0; i < kScanItems; ++i) {
    const long long g = t0 + i;
    bool limited;
    B[i] = g < a.nb ? a.counts[g] : 0;
    K[i] = kept_of(B[i], a.alpha, a.P, a.minSize, &limited);
    sc += B[i];
    sk += K[i];
  }
  long long tc, tk;
  long long ec = block_exclusive_scan(sc, tmp, &tc) + (long long)a.blk_cnt[blockIdx.x];
  long long ek = block_exclusive_scan(sk, tmp, &tk) + (long long)a.blk_kept[blockIdx.x];
  for (int i = 0; i < kScanItems; ++i) {
    const long long g = t0 + i;
    if (g < a.nb) {
      a.segstart[g] = (uint32_t)ec;
      a.off[g] = (uint32_t)ek;
    }
    ec += B[i];
    ek += K[i];
  }
}

// ---------------------------------------------------------------- radix sort
constexpr int kRsThreads = 256;
constexpr int kRsItems = 16;
constexpr int kRsTile = kRsThreads * kRsItems;

__global__ void __launch_bounds__(kRsThreads) k_rs_hist(const uint64_t* __restrict__ keys, long long N, int shift,
                                                         uint32_t* __restrict__ hist, int ntiles) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const long long base = (long long)blockIdx.x * kRsTile;
#pragma unroll 4
  for (int i = 0; i < kRsItems; ++i) {
    const long long idx = base + (long long)i * kRsThreads + threadIdx.x;
    if (idx < N) atomicAdd(&h[(uint32_t)(keys[idx] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[(size_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// one block per digit: exclusive scan over the tiles of that digit
__global__ void __launch_bounds__(1024) k_rs_scan(uint32_t* __restrict__ hist, int ntiles,
                                                  uint32_t* __restrict__ digit_total) {
  __shared__ long long tmp[32];
  uint32_t* h = hist + (size_t)blockIdx.x * ntiles;
  const int per = (ntiles + 1023) / 1024;
  const int t0 = threadIdx.x * per;
  long long s = 0;
  for (int i = 0; i < per; ++i)
    if (t0 + i < ntiles) s += h[t0 + i];
  long long total;
  long long run = block_exclusive_scan(s, tmp, &total);
  for (int i = 0; i < per; ++i)
    if (t0 + i < ntiles) {
      const uint32_t v = h[t0 + i];
      h[t0 + i] = (uint32_t)run;
      run += v;
    }
  if (threadIdx.x == 0) digit_total[blockIdx.x] = (uint32_t)total;
}

__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const uint64_t* __restrict__ kin,
                                                            const uint32_t* __restrict__ vin,
                                                            uint64_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                            long long N, int shift, const uint32_t* __restrict__ hist,
                                                            int ntiles, const uint32_t* __restrict__ digit_total) {
  __shared__ long long tmp[32];
  __shared__ uint32_t base[256];
  __shared__ uint32_t wcnt[kRsThreads / 32][257];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  long long tot;
  const long long dbase = block_exclusive_scan((long long)digit_total[tid], tmp, &tot);
  base[tid] = (uint32_t)dbase + hist[(size_t)tid * ntiles + blockIdx.x];
  for (int w = 0; w < kRsThreads / 32; ++w) wcnt[w][tid] = 0;
  if (tid == 0)
    for (int w = 0; w < kRsThreads / 32; ++w) wcnt[w][256] = 0;
  __syncthreads();
  const long long tbase = (long long)blockIdx.x * kRsTile;
  const unsigned lt = (1u << lane) - 1u;
  for (int it = 0; it < kRsItems; ++it) {
    const long long idx = tbase + (long long)it * kRsThreads + tid;
    const bool valid = idx < N;
    const uint64_t k = valid ? kin[idx] : 0ull;
    const uint32_t v = valid ? vin[idx] : 0u;
    const uint32_t dg = valid ? ((uint32_t)(k >> shift) & 255u) : 256u;
    const unsigned peers = __match_any_sync(kFullMask, dg);
    const int rank = __popc(peers & lt);
    if (valid && lane == __ffs(peers) - 1) wcnt[warp][dg] = __popc(peers);
    __syncthreads();
    if (valid) {
      uint32_t o = base[dg];
      for (int w = 0; w < warp; ++w) o += wcnt[w][dg];
      kout[o + rank] = k;
      vout[o + rank] = v;
    }
    __syncthreads();
    uint32_t s = 0;
    for (int w = 0; w < kRsThreads / 32; ++w) {
      s += wcnt[w][tid];
      wcnt[w][tid] = 0;
    }
    base[tid] += s;
    __syncthreads();
  }
}

// ---------------------------------------------------------------- compaction
struct CompactArgs {
  const uint64_t* keys;  // sorted
  const uint32_t* vals;
  long long N;
  const uint32_t* counts;  // global [L*NB]
  const uint32_t* segstart;  // chunk-local
  const uint32_t* off;       // global
  unsigned long long gbase;  // first global bucket of the chunk
  float alpha;
  int P, minSize;
  int exact_order;
  int32_t* ids;
  uint32_t* flags;       // chunk-local, one per bucket
  uint32_t* repair;      // chunk-local bucket list
  unsigned int* n_repair;
};

__global__ void k_compact(CompactArgs a) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  const uint64_t key = a.keys[i];
  const uint32_t grel = (uint32_t)(key >> 32);
  const unsigned long long g = a.gbase + grel;
  const uint32_t B = a.counts[g];
  bool limited;
  const uint32_t kp = kept_of(B, a.alpha, a.P, a.minSize, &limited);
  const uint32_t rank = (uint32_t)(i - (long long)a.segstart[grel]);
  if (rank < kp) {
    a.ids[a.off[g] + rank] = (int32_t)a.vals[i];
    if (rank + 1 < B && (rank + 1 == kp || a.exact_order)) {
      if ((uint32_t)a.keys[i + 1] == (uint32_t)key) {  // equal score next to a kept entry
        if (atomicOr(a.flags + grel, 1u) == 0u) {
          const unsigned slot = atomicAdd(a.n_repair, 1u);
          a.repair[slot] = grel;
        }
      }
    }
  }
}

// ---------------------------------------------------------------- tie repair
constexpr int kRepairSmemEntries = 4096;  // 32 KB of static shared memory

struct RepairArgs {
  const uint64_t* keys;  // sorted
  const uint32_t* vals;
  uint32_t* sk;          // scratch ids   (alternate sort buffer, same positions)
  uint32_t* sv;          // scratch scores
  const uint32_t* counts;
  const uint32_t* segstart;
  const uint32_t* off;
  unsigned long long gbase;
  float alpha;
  int P, minSize;
  const uint32_t* repair;
  const unsigned int* n_repair;
  int32_t* ids;
};

// One block per bucket: put the bucket's entries back in push order (ascending
// id, FalconnPP.cpp:75 / :200), then thread 0 replays the priority_queue pushes
// and the first iLimit pops (FalconnPP.cpp:226-230).
__global__ void __launch_bounds__(256) k_repair(RepairArgs a) {
  __shared__ uint32_t s_id[kRepairSmemEntries];
  __shared__ uint32_t s_sc[kRepairSmemEntries];
  const unsigned nrep = *a.n_repair;
  for (unsigned r = blockIdx.x; r < nrep; r += gridDim.x) {
    const uint32_t grel = a.repair[r];
    const unsigned long long g = a.gbase + grel;
    const uint32_t B = a.counts[g];
    bool limited;
    const uint32_t kp = kept_of(B, a.alpha, a.P, a.minSize, &limited);
    const uint32_t s0 = a.segstart[grel];
    const bool in_smem = B <= (uint32_t)kRepairSmemEntries;
    uint32_t* pid = in_smem ? s_id : a.sk + s0;
    uint32_t* psc = in_smem ? s_sc : a.sv + s0;
    for (uint32_t i = threadIdx.x; i < B; i += blockDim.x) {
      pid[i] = a.vals[s0 + i];
      psc[i] = ord_key_inv_dev(~(uint32_t)a.keys[s0 + i]);  // float bits of the score
    }
    __syncthreads();
    block_bitonic_sort_u32(pid, psc, (int)B);
    if (threadIdx.x == 0) {
      float* hv = reinterpret_cast<float*>(psc);
      int* hi = reinterpret_cast<int*>(pid);
      int n = 0;
      for (uint32_t i = 0; i < B; ++i) heap_push<false, int>(hv, hi, n, hv[i], hi[i]);
      int32_t* out = a.ids + a.off[g];
      for (uint32_t j = 0; j < kp; ++j) {
        out[j] = hi[0];
        heap_pop<false, int>(hv, hi, n);
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- host side
template <int FHT>
static cudaError_t launch_hash(const HashArgs& a, int nsm, cudaStream_t s) {
  const size_t smem = HashSmem<FHT>::bytes;
  cudaError_t e = cudaFuncSetAttribute(k_build_hash<FHT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_build_hash<FHT>, 128, smem);
  if (e != cudaSuccess) return e;
  const long long groups_needed = (a.n + HashSmem<FHT>::GROUPS - 1) / HashSmem<FHT>::GROUPS;
  const long long grid = std::max(1LL, std::min<long long>((long long)nsm * std::max(per_sm, 1), groups_needed));
  k_build_hash<FHT><<<(unsigned)grid, 128, smem, s>>>(a);
  return cudaGetLastError();
}

static cudaError_t dispatch_hash(int fht, const HashArgs& a, int nsm, cudaStream_t s) {
  switch (fht) {
    case 2: return launch_hash<2>(a, nsm, s);
    case 4: return launch_hash<4>(a, nsm, s);
    case 8: return launch_hash<8>(a, nsm, s);
    case 16: return launch_hash<16>(a, nsm, s);
    case 32: return launch_hash<32>(a, nsm, s);
    case 64: return launch_hash<64>(a, nsm, s);
    case 128: return launch_hash<128>(a, nsm, s);
    case 256: return launch_hash<256>(a, nsm, s);
    case 512: return launch_hash<512>(a, nsm, s);
    case 1024: return launch_hash<1024>(a, nsm, s);
    default: return cudaErrorInvalidValue;
  }
}

static double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

void free_index(DeviceIndex& di) {
  cudaFree(di.Xc);
  cudaFree(di.center);
  cudaFree(di.flips);
  cudaFree(di.tflips);
  cudaFree(di.bucket_off);
  cudaFree(di.ids);
  cudaFree(di.Xlp);
  cudaFree(di.Xlp_scale);
  di = DeviceIndex();
}

int upload_flips(const Params& P, const HostBits& bits, DeviceIndex& di, cudaStream_t s, Error& err) {
  const int L = P.n_tables, F = P.fhtDim;
  const int WORDS = F < 32 ? 1 : F / 32;
  std::vector<uint32_t> hflips((size_t)2 * L * 3 * WORDS, 0u);
  std::vector<uint32_t> htflips;
  for (int layer = 0; layer < 2; ++layer) {
    const std::vector<uint8_t>& b = layer == 0 ? bits.b1 : bits.b2;
    for (int l = 0; l < L; ++l)
      for (int r = 0; r < 3; ++r)
        for (int i = 0; i < F; ++i) {
          const uint8_t bit = b[(size_t)l * 3 * F + (size_t)r * F + i];
          if (bit == 0) hflips[(((size_t)layer * L + l) * 3 + r) * WORDS + i / 32] |= 1u << (i % 32);
        }
  }
  FPP_CUDA(fpp::dev_malloc(&di.flips, sizeof(uint32_t) * hflips.size()));
  FPP_CUDA(cudaMemcpyAsync(di.flips, hflips.data(), sizeof(uint32_t) * hflips.size(), cudaMemcpyHostToDevice, s));
  if (F == 256) {
    // the tensor-core rotation (batched low-precision form) reads round 2's
    // signs in the transposed view: bit 16k + n of its words is the sign of
    // position 16n + k
    htflips = hflips;
    for (size_t v = 0; v < (size_t)2 * L; ++v) {
      const uint32_t* src = hflips.data() + (v * 3 + 1) * WORDS;
      uint32_t* dst = htflips.data() + (v * 3 + 1) * WORDS;
      for (int w = 0; w < WORDS; ++w) dst[w] = 0u;
      for (int pp = 0; pp < 256; ++pp) {
        const int p0 = 16 * (pp & 15) + (pp >> 4);
        if ((src[p0 >> 5] >> (p0 & 31)) & 1u) dst[pp >> 5] |= 1u << (pp & 31);
      }
    }
    FPP_CUDA(fpp::dev_malloc(&di.tflips, sizeof(uint32_t) * htflips.size()));
    FPP_CUDA(cudaMemcpyAsync(di.tflips, htflips.data(), sizeof(uint32_t) * htflips.size(), cudaMemcpyHostToDevice,
                             s));
  }
  // the host vectors go out of scope here
  FPP_CUDA(cudaStreamSynchronize(s));
  return kOk;
fail:
  return err.code;
}

int build_index(const Params& P, const float* X, bool x_on_device, const HostBits& bits,
                const BuildOptions& opt, DeviceIndex& di, BuildStats& st, cudaStream_t s, Error& err,
                int32_t* dump_codes, float* dump_scores) {
  const auto t_start = std::chrono::steady_clock::now();
  const long long n = P.n_points;
  const int d = P.n_features, L = P.n_tables, D = P.n_proj, F = P.fhtDim, IP = P.iProbes;
  const uint32_t NB = 4u * (uint32_t)D * (uint32_t)D;
  const int ld = (d + 3) & ~3;
  int log2D = 0;
  while ((1 << log2D) < D) ++log2D;

  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);

  float* Xstage = nullptr;
  float* part = nullptr;
  int* d_bad = nullptr;
  uint32_t* counts = nullptr;
  uint64_t* keys[2] = {nullptr, nullptr};
  uint32_t* vals[2] = {nullptr, nullptr};
  uint32_t* hist = nullptr;
  uint32_t* digit_total = nullptr;
  uint32_t* segstart = nullptr;
  uint32_t* flags = nullptr;
  uint32_t* repair = nullptr;
  unsigned int* n_repair = nullptr;
  unsigned long long* blk_cnt = nullptr;
  unsigned long long* blk_kept = nullptr;
  unsigned long long* d_base = nullptr;
  unsigned int* d_maxkept = nullptr;
  unsigned long long* d_limited = nullptr;
  int32_t* ids_cap = nullptr;
  uint64_t ids_capacity = 0;
  int h_bad = 0;
  unsigned long long h_base = 0;
  long long tables_per_chunk = 0;
  const long long entry_cap = 1LL << 27;
  long long max_entries = 0;
  long long nb_chunk_max = 0;
  long long nblk_max = 0;
  int ntiles_max = 0;
  const long long nchunks_c = (n + kCenterChunk - 1) / kCenterChunk;

  free_index(di);
  di.ld = ld;

  // 1. centre
  {
    auto t0 = std::chrono::steady_clock::now();
    const float* Xd = X;
    if (!x_on_device) {
      FPP_CUDA(fpp::dev_malloc(&Xstage, sizeof(float) * n * d));
      FPP_CUDA(cudaMemcpyAsync(Xstage, X, sizeof(float) * n * d, cudaMemcpyHostToDevice, s));
      Xd = Xstage;
    }
    FPP_CUDA(fpp::dev_malloc(&di.Xc, sizeof(float) * n * ld));
    FPP_CUDA(fpp::dev_malloc(&di.center, sizeof(float) * d));
    FPP_CUDA(fpp::dev_malloc(&part, sizeof(float) * nchunks_c * d));
    FPP_CUDA(fpp::dev_malloc(&d_bad, sizeof(int)));
    FPP_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), s));
    dim3 g1((unsigned)nchunks_c, (unsigned)((d + 255) / 256));
    k_center_partial<<<g1, 256, 0, s>>>(Xd, n, d, part);
    k_center_final<<<(d + 255) / 256, 256, 0, s>>>(part, nchunks_c, n, d, di.center);
    k_center_apply<<<(unsigned)std::max(1, nsm * 8), 256, 0, s>>>(Xd, n, d, ld, di.center, di.Xc, d_bad);
    FPP_CUDA(cudaGetLastError());
    FPP_CUDA(cudaMemcpyAsync(&h_bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    FPP_CUDA(cudaStreamSynchronize(s));
    cudaFree(Xstage);
    Xstage = nullptr;
    if (h_bad) {
      err.code = kErrNonFinite;
      err.msg = "build: the dataset contains NaN or infinite values";
      goto fail;
    }
    st.ms_center = ms_since(t0);
  }

  // 2. random signs -> flip words [2][L][3][WORDS]
  if (upload_flips(P, bits, di, s, err) != kOk) goto fail;

  // 3. hash + sort + compact, a chunk of tables at a time
  tables_per_chunk = opt.tables_per_chunk > 0 ? opt.tables_per_chunk
                                               : std::max(1LL, std::min<long long>(L, entry_cap / std::max(1LL, n * IP)));
  tables_per_chunk = std::min<long long>(tables_per_chunk, L);
  max_entries = tables_per_chunk * n * IP;
  nb_chunk_max = tables_per_chunk * (long long)NB;
  nblk_max = (nb_chunk_max + kScanTile - 1) / kScanTile;
  ntiles_max = (int)((max_entries + kRsTile - 1) / kRsTile);
  if (max_entries >= (1LL << 32) || nb_chunk_max >= (1LL << 32)) {
    err.code = kErrUnsupported;
    err.msg = "build: too many entries per table chunk";
    goto fail;
  }
  FPP_CUDA(fpp::dev_malloc(&counts, sizeof(uint32_t) * (size_t)L * NB));
  FPP_CUDA(cudaMemsetAsync(counts, 0, sizeof(uint32_t) * (size_t)L * NB, s));
  FPP_CUDA(fpp::dev_malloc(&di.bucket_off, sizeof(uint32_t) * ((size_t)L * NB + 1)));
  for (int i = 0; i < 2; ++i) {
    FPP_CUDA(fpp::dev_malloc(&keys[i], sizeof(uint64_t) * std::max(1LL, max_entries)));
    FPP_CUDA(fpp::dev_malloc(&vals[i], sizeof(uint32_t) * std::max(1LL, max_entries)));
  }
  FPP_CUDA(fpp::dev_malloc(&hist, sizeof(uint32_t) * 256 * (size_t)std::max(1, ntiles_max)));
  FPP_CUDA(fpp::dev_malloc(&digit_total, sizeof(uint32_t) * 256));
  FPP_CUDA(fpp::dev_malloc(&segstart, sizeof(uint32_t) * nb_chunk_max));
  FPP_CUDA(fpp::dev_malloc(&flags, sizeof(uint32_t) * nb_chunk_max));
  FPP_CUDA(fpp::dev_malloc(&repair, sizeof(uint32_t) * nb_chunk_max));
  FPP_CUDA(fpp::dev_malloc(&n_repair, sizeof(unsigned int)));
  FPP_CUDA(fpp::dev_malloc(&blk_cnt, sizeof(unsigned long long) * nblk_max));
  FPP_CUDA(fpp::dev_malloc(&blk_kept, sizeof(unsigned long long) * nblk_max));
  FPP_CUDA(fpp::dev_malloc(&d_base, sizeof(unsigned long long)));
  FPP_CUDA(fpp::dev_malloc(&d_maxkept, sizeof(unsigned int)));
  FPP_CUDA(fpp::dev_malloc(&d_limited, sizeof(unsigned long long)));
  FPP_CUDA(cudaMemsetAsync(d_base, 0, sizeof(unsigned long long), s));
  FPP_CUDA(cudaMemsetAsync(d_maxkept, 0, sizeof(unsigned int), s));
  FPP_CUDA(cudaMemsetAsync(d_limited, 0, sizeof(unsigned long long), s));

  for (long long l0 = 0; l0 < L; l0 += tables_per_chunk) {
    const long long l1 = std::min<long long>(L, l0 + tables_per_chunk);
    const long long Ne = (l1 - l0) * n * IP;
    const long long nbc = (l1 - l0) * (long long)NB;
    auto t0 = std::chrono::steady_clock::now();
    HashArgs ha;
    ha.Xc = di.Xc;
    ha.ld = ld;
    ha.n = (int)n;
    ha.d = d;
    ha.flips = di.flips;
    ha.L = L;
    ha.l0 = (int)l0;
    ha.l1 = (int)l1;
    ha.D = D;
    ha.log2D = log2D;
    ha.P = IP;
    ha.NB = NB;
    ha.keys = keys[0];
    ha.vals = vals[0];
    ha.counts = counts;
    ha.dump_codes = dump_codes;
    ha.dump_scores = dump_scores;
    FPP_CUDA(dispatch_hash(F, ha, nsm, s));
    FPP_CUDA(cudaStreamSynchronize(s));
    st.ms_hash += ms_since(t0);

    // bucket limits and CSR offsets of this chunk
    t0 = std::chrono::steady_clock::now();
    ScanArgs sa;
    sa.counts = counts + l0 * NB;
    sa.nb = nbc;
    sa.alpha = P.bucket_scale;
    sa.P = IP;
    sa.minSize = P.bucket_minSize;
    sa.segstart = segstart;
    sa.off = di.bucket_off + l0 * NB;
    sa.blk_cnt = blk_cnt;
    sa.blk_kept = blk_kept;
    sa.base = d_base;
    sa.max_kept = d_maxkept;
    sa.n_limited = d_limited;
    const long long nblk = (nbc + kScanTile - 1) / kScanTile;
    k_scan_reduce<<<(unsigned)nblk, kScanThreads, 0, s>>>(sa);
    k_scan_blocks<<<1, kScanThreads, 0, s>>>(sa, nblk);
    k_scan_down<<<(unsigned)nblk, kScanThreads, 0, s>>>(sa);
    FPP_CUDA(cudaGetLastError());
    FPP_CUDA(cudaMemcpyAsync(&h_base, d_base, sizeof(h_base), cudaMemcpyDeviceToHost, s));
    FPP_CUDA(cudaStreamSynchronize(s));
    if (h_base >= (1ULL << 32)) {
      err.code = kErrUnsupported;
      err.msg = "build: more than 2^32-1 stored ids (the bucket positions are 32-bit, src/FalconnPP.h:33)";
      goto fail;
    }
    if (h_base > ids_capacity) {  // grow the 1D table
      uint64_t cap = std::max<uint64_t>(h_base, ids_capacity * 3 / 2);
      cap = std::min<uint64_t>(std::max<uint64_t>(cap, h_base), std::max<uint64_t>(h_base, (uint64_t)L * n * IP));
      int32_t* nids = nullptr;
      FPP_CUDA(fpp::dev_malloc(&nids, sizeof(int32_t) * cap));
      if (ids_cap && di.n_ids)
        FPP_CUDA(cudaMemcpyAsync(nids, ids_cap, sizeof(int32_t) * di.n_ids, cudaMemcpyDeviceToDevice, s));
      FPP_CUDA(cudaStreamSynchronize(s));
      cudaFree(ids_cap);
      ids_cap = nids;
      ids_capacity = cap;
    }
    di.n_ids = h_base;
    st.ms_csr += ms_since(t0);

    // sort the chunk's entries by (bucket, score desc), stable
    t0 = std::chrono::steady_clock::now();
    int bbits = 0;
    while ((1LL << bbits) < nbc) ++bbits;
    const int total_bits = 32 + bbits;
    const int ntiles = (int)((Ne + kRsTile - 1) / kRsTile);
    int cur = 0;
    for (int shift = 0; shift < total_bits; shift += 8) {
      k_rs_hist<<<ntiles, kRsThreads, 0, s>>>(keys[cur], Ne, shift, hist, ntiles);
      k_rs_scan<<<256, 1024, 0, s>>>(hist, ntiles, digit_total);
      k_rs_scatter<<<ntiles, kRsThreads, 0, s>>>(keys[cur], vals[cur], keys[cur ^ 1], vals[cur ^ 1], Ne, shift, hist,
                                                 ntiles, digit_total);
      cur ^= 1;
    }
    FPP_CUDA(cudaGetLastError());
    FPP_CUDA(cudaStreamSynchronize(s));
    st.ms_sort += ms_since(t0);

    t0 = std::chrono::steady_clock::now();
    FPP_CUDA(cudaMemsetAsync(flags, 0, sizeof(uint32_t) * nbc, s));
    FPP_CUDA(cudaMemsetAsync(n_repair, 0, sizeof(unsigned int), s));
    CompactArgs ca;
    ca.keys = keys[cur];
    ca.vals = vals[cur];
    ca.N = Ne;
    ca.counts = counts;
    ca.segstart = segstart;
    ca.off = di.bucket_off;
    ca.gbase = (unsigned long long)l0 * NB;
    ca.alpha = P.bucket_scale;
    ca.P = IP;
    ca.minSize = P.bucket_minSize;
    ca.exact_order = opt.exact_bucket_order ? 1 : 0;
    ca.ids = ids_cap;
    ca.flags = flags;
    ca.repair = repair;
    ca.n_repair = n_repair;
    k_compact<<<(unsigned)((Ne + 255) / 256), 256, 0, s>>>(ca);
    FPP_CUDA(cudaGetLastError());
    unsigned int h_rep = 0;
    FPP_CUDA(cudaMemcpyAsync(&h_rep, n_repair, sizeof(h_rep), cudaMemcpyDeviceToHost, s));
    FPP_CUDA(cudaStreamSynchronize(s));
    if (h_rep) {
      RepairArgs ra;
      ra.keys = keys[cur];
      ra.vals = vals[cur];
      ra.sk = reinterpret_cast<uint32_t*>(keys[cur ^ 1]);
      ra.sv = vals[cur ^ 1];
      ra.counts = counts;
      ra.segstart = segstart;
      ra.off = di.bucket_off;
      ra.gbase = (unsigned long long)l0 * NB;
      ra.alpha = P.bucket_scale;
      ra.P = IP;
      ra.minSize = P.bucket_minSize;
      ra.repair = repair;
      ra.n_repair = n_repair;
      ra.ids = ids_cap;
      k_repair<<<std::min<unsigned>(h_rep, (unsigned)nsm * 4), 256, 0, s>>>(ra);
      FPP_CUDA(cudaGetLastError());
      FPP_CUDA(cudaStreamSynchronize(s));
    }
    st.n_repaired += h_rep;
    st.ms_csr += ms_since(t0);
  }
  {
    const uint32_t last = (uint32_t)h_base;
    FPP_CUDA(cudaMemcpyAsync(di.bucket_off + (size_t)L * NB, &last, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    unsigned long long lim = 0;
    FPP_CUDA(cudaMemcpyAsync(&di.max_kept, d_maxkept, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    FPP_CUDA(cudaMemcpyAsync(&lim, d_limited, sizeof(lim), cudaMemcpyDeviceToHost, s));
    FPP_CUDA(cudaStreamSynchronize(s));
    st.n_limited = (long long)lim;
    st.points_per_table = (double)h_base / (double)n / (double)L;
  }
  if (ids_cap == nullptr) FPP_CUDA(fpp::dev_malloc(&ids_cap, sizeof(int32_t)));
  di.ids = ids_cap;
  ids_cap = nullptr;

  cudaFree(part);
  cudaFree(d_bad);
  cudaFree(counts);
  for (int i = 0; i < 2; ++i) {
    cudaFree(keys[i]);
    cudaFree(vals[i]);
  }
  cudaFree(hist);
  cudaFree(digit_total);
  cudaFree(segstart);
  cudaFree(flags);
  cudaFree(repair);
  cudaFree(n_repair);
  cudaFree(blk_cnt);
  cudaFree(blk_kept);
  cudaFree(d_base);
  cudaFree(d_maxkept);
  cudaFree(d_limited);
  st.ms_total = ms_since(t_start);
  return kOk;

fail:
  cudaStreamSynchronize(s);
  cudaFree(Xstage);
  cudaFree(part);
  cudaFree(d_bad);
  cudaFree(counts);
  for (int i = 0; i < 2; ++i) {
    cudaFree(keys[i]);
    cudaFree(vals[i]);
  }
  cudaFree(hist);
  cudaFree(digit_total);
  cudaFree(segstart);
  cudaFree(flags);
  cudaFree(repair);
  cudaFree(n_repair);
  cudaFree(blk_cnt);
  cudaFree(blk_kept);
  cudaFree(d_base);
  cudaFree(d_maxkept);
  cudaFree(d_limited);
  cudaFree(ids_cap);
  free_index(di);
  return err.code;
}

}  // namespace fpp
