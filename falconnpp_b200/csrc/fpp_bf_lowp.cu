// fpp_bf_lowp.cu — brute-force maximum-inner-product search over the index's
// BF16 or FP8-E4M3 row copies on the tcgen05 tensor cores, with the top-R
// selection fused into the accumulator epilogue and an exact FP32 re-score of
// the shortlist (the block rerank of the precision form; model: BF::mips_topK,
// src/BF.cpp:17-86, an exact GEMV + size-k min-heap per query).
//
// k_bf_lowp — one CTA per (query tile of 128, split of the rows):
//   warp 0      TMA producer: the query tile once, then row tiles of 128 into
//               a ring of shared-memory stages (128-byte swizzle, K-major);
//   warp 1      owns TMEM (256 columns: two 128-column accumulators) and
//               issues tcgen05.mma (M = 128 queries, N = 128 rows, K = 16
//               BF16 / 32 E4M3 per instruction, FP32 accumulate), committing
//               each tile to the stage's "empty" and the accumulator's "full"
//               barrier;
//   warps 2..5  epilogue: thread = one query (TMEM lane), reads its 128
//               scores with tcgen05.ld, applies the FP8 row/query scales and
//               keeps its own size-R min-heap of 64-bit keys (score, ~id), so
//               the kept set is the split's top R by (score desc, id asc)
//               even among equal scores (global scratch, touched only on the
//               rare insertions at or above the heap's minimum).
// The CTAs of one split run side by side over the same rows, so a row tile
// comes from HBM once and from L2 for the other query tiles.
//
// k_bf_merge — one block per query: the S heaps' candidates, the best R by
// the low-precision score (ties: smaller id), their exact FP32 inner
// products in the canonical dot order of the query path, and the top k by
// (score desc, id asc).
//
// Every mbarrier wait gives up after a bounded number of polls; a CTA that
// gives up raises the status word, lets its copies and MMAs drain (bounded
// again), frees its TMEM and exits.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/falconnpp_b200.h"
#include "fpp_batch.h"
#include "fpp_device.cuh"
#include "fpp_handle.h"
#include "fpp_rows.cuh"

namespace fpp {
namespace {

constexpr int kTile = 128;          // queries per CTA (MMA M) and rows per tile (MMA N)
constexpr int kBoxBytes = 128;      // K bytes per TMA box (the 128-byte swizzle span)
constexpr int kKPadBytes = 512;     // K bytes covered (BF16: d <= 256; E4M3: d <= 512)
constexpr int kBoxTileBytes = kTile * kBoxBytes;  // 16 KB: 128 rows of one box
constexpr int kThreads = 192;
constexpr int kMaxR = 256;          // shortlist per query
constexpr int kMaxRS = 32;          // per-split heap in shared memory: 128 queries x 32 keys = 32 KB
constexpr uint32_t kMaxPolls = 1u << 24;
constexpr int kTmemCols = 256;

template <int MODE>
struct BfCfg {
  static constexpr int esize = MODE == kRowsBF16 ? 2 : 1;
  static constexpr int box_elems = kBoxBytes / esize;
};

struct BfArgs {
  int n, nq, d, kbytes;        // kbytes: K bytes actually multiplied (multiple of 32)
  int boxes;                   // TMA boxes per tile (kbytes rounded up to 128)
  int stages;
  int rows_per_split, splits, qtiles;
  int R;                       // shortlist per query (merge)
  int rs;                      // per-split heap size, min(R, kMaxRS)
  const float* xscale;         // FP8 per-row scales (nullable for BF16)
  const float* qscale;         // FP8 per-query scales
  unsigned long long* heap;    // [nq][splits][rs] keys (ord(score) << 32) | ~id
  int* heap_n;                 // [nq][splits]
  unsigned* status;            // bit 0: a CTA gave up waiting
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: false once the CTA's abort flag is up or the poll budget is
// spent (then it raises the flag itself).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
  for (uint32_t it = 0; it < kMaxPolls; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 255u) == 255u && *abort_flag) return false;
  }
  *abort_flag = 1;
  return false;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

// K-major operand in the canonical 128-byte-swizzle layout: 8-row atoms of
// 128-byte rows, atoms 1024 bytes apart (stride byte offset), version 1.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// kind::f16 (BF16 x BF16) or kind::f8f6f4 (E4M3 x E4M3), FP32 accumulator,
// both operands K-major, M = N = 128.
template <int MODE>
__host__ __device__ constexpr uint32_t umma_idesc() {
  return (1u << 4) | (MODE == kRowsBF16 ? ((1u << 7) | (1u << 10)) : 0u) | ((uint32_t)(kTile >> 3) << 17) |
         ((uint32_t)(kTile >> 4) << 24);
}

template <int MODE>
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
  const uint32_t idesc = umma_idesc<MODE>();
  if constexpr (MODE == kRowsBF16) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n}\n"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u));
  } else {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n}\n"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u));
  }
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// size-R min-heap of keys (larger key = better candidate), slot j at h[j * st]
__device__ __forceinline__ void key_heap_offer_strided(unsigned long long* h, int st, int& n, int R, unsigned long long key) {
  int i;
  if (n < R) {
    i = n++;
    while (i > 0) {
      const int p = (i - 1) >> 1;
      const unsigned long long hp = h[p * st];
      if (hp <= key) break;
      h[i * st] = hp;
      i = p;
    }
    h[i * st] = key;
    return;
  }
  if (key <= h[0]) return;
  i = 0;
  for (;;) {
    int c = 2 * i + 1;
    if (c >= n) break;
    unsigned long long hc = h[c * st];
    if (c + 1 < n) {
      const unsigned long long h2 = h[(c + 1) * st];
      if (h2 < hc) {
        hc = h2;
        ++c;
      }
    }
    if (hc >= key) break;
    h[i * st] = hc;
    i = c;
  }
  h[i * st] = key;
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

template <int MODE>
__global__ void __launch_bounds__(kThreads, 1)
    k_bf_lowp(const __grid_constant__ CUtensorMap qmap, const __grid_constant__ CUtensorMap xmap, BfArgs a) {
  using C = BfCfg<MODE>;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte alignment of the operand tiles (the swizzle atom)
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int tile_bytes = a.boxes * kBoxTileBytes;
  unsigned char* q_smem = base;
  unsigned char* x_smem = base + tile_bytes;
  unsigned long long* heap_smem = reinterpret_cast<unsigned long long*>(x_smem + (size_t)a.stages * tile_bytes);
  uint64_t* bars = reinterpret_cast<uint64_t*>(heap_smem + (size_t)kTile * a.rs);
  // bars: [0] q_full, [1..S] full, [S+1..2S] empty, [2S+1..2S+2] acc full, [2S+3..2S+4] acc empty
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * a.stages + 5);
  __shared__ int s_abort;

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int S = a.stages;
  const int qt = blockIdx.x % a.qtiles;
  const int split = blockIdx.x / a.qtiles;
  const int q0 = qt * kTile;
  const int r0 = split * a.rows_per_split;
  const int r1 = min(a.n, r0 + a.rows_per_split);
  const int ntiles = r1 > r0 ? (r1 - r0 + kTile - 1) / kTile : 0;
  const int ksteps = a.kbytes / 32;

  auto bar = [&](int i) { return smem_u32(bars + i); };
  if (threadIdx.x == 0) {
    s_abort = 0;
    mbar_init(bar(0), 1);
    for (int s = 0; s < S; ++s) {
      mbar_init(bar(1 + s), 1);
      mbar_init(bar(1 + S + s), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(bar(2 * S + 1 + b), 1);
      mbar_init(bar(2 * S + 3 + b), 4);  // one arrival per epilogue warp
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  volatile int* abort_flag = &s_abort;

  if (warp == 0) {
    // ---- producer
    if (lane == 0) {
      int issued = 0;
      bool ok = true;
      mbar_expect_tx(bar(0), (uint32_t)tile_bytes);
      for (int bx = 0; bx < a.boxes; ++bx)
        tma_load_2d(smem_u32(q_smem + bx * kBoxTileBytes), &qmap, bx * C::box_elems, q0, bar(0));
      for (int i = 0; i < ntiles && ok; ++i) {
        const int s = i % S;
        ok = mbar_wait(bar(1 + S + s), ((i / S) & 1) ^ 1, abort_flag);
        if (!ok) break;
        mbar_expect_tx(bar(1 + s), (uint32_t)tile_bytes);
        unsigned char* dst = x_smem + (size_t)s * tile_bytes;
        for (int bx = 0; bx < a.boxes; ++bx)
          tma_load_2d(smem_u32(dst + bx * kBoxTileBytes), &xmap, bx * C::box_elems, r0 + i * kTile, bar(1 + s));
        issued = i + 1;
      }
      // let every copy issued land before the CTA can exit (bounded)
      mbar_wait(bar(0), 0, abort_flag);
      for (int i = max(0, issued - S); i < issued; ++i) {
        volatile int never = 0;
        mbar_wait(bar(1 + i % S), (i / S) & 1, &never);
      }
    }
  } else if (warp == 1) {
    // ---- MMA issuer
    if (lane == 0) {
      bool ok = mbar_wait(bar(0), 0, abort_flag);
      const uint32_t qa = smem_u32(q_smem);
      int issued = 0;
      for (int i = 0; i < ntiles && ok; ++i) {
        const int s = i % S;
        const int b = i & 1;
        ok = mbar_wait(bar(2 * S + 3 + b), ((i >> 1) & 1) ^ 1, abort_flag);
        if (!ok) break;
        ok = mbar_wait(bar(1 + s), (i / S) & 1, abort_flag);
        if (!ok) break;
        tc_fence_after();
        const uint32_t xa = smem_u32(x_smem + (size_t)s * tile_bytes);
        for (int t = 0; t < ksteps; ++t) {
          const uint32_t off = (uint32_t)((t >> 2) * kBoxTileBytes + (t & 3) * 32);
          umma<MODE>(tmem + (uint32_t)(b * kTile), umma_desc_sw128(qa + off), umma_desc_sw128(xa + off),
                     t > 0 ? 1u : 0u);
        }
        umma_commit(bar(1 + S + s));
        umma_commit(bar(2 * S + 1 + b));
        issued = i + 1;
      }
      if (issued > 0) {  // the last tile's MMAs complete before TMEM is freed
        volatile int never = 0;
        mbar_wait(bar(2 * S + 1 + ((issued - 1) & 1)), ((issued - 1) >> 1) & 1, &never);
      }
    }
  } else {
    // ---- epilogue: thread = query q of the tile
    const int quad = warp & 3;  // the TMEM lanes this warp may read
    const int ql = quad * 32 + lane;
    const int q = q0 + ql;
    const bool live = q < a.nq;
    const int RS = a.rs;
    // the split's top RS keys of this query in shared memory, slot j at
    // hk[j * kTile] (consecutive queries in consecutive words)
    unsigned long long* hk = heap_smem + ql;
    int hn = 0;
    float thr = -INFINITY;  // score of the heap's minimum once the heap is full
    const float qs = (MODE == kRowsFP8 && live) ? a.qscale[q] : 1.0f;
    for (int i = 0; i < ntiles; ++i) {
      const int b = i & 1;
      if (!mbar_wait(bar(2 * S + 1 + b), (i >> 1) & 1, abort_flag)) break;
      tc_fence_after();
      float v[4][32];
      const uint32_t taddr = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(b * kTile);
#pragma unroll
      for (int c = 0; c < 4; ++c) tmem_ld32(taddr + c * 32, v[c]);
      tmem_wait_ld();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(bar(2 * S + 3 + b));
      const int x0 = r0 + i * kTile;
      const int nvalid = min(kTile, r1 - x0);
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        if (MODE == kRowsFP8) {
          // lane t holds the scale of column c * 32 + t; column j's is shuffled in
          const int xr = x0 + c * 32 + lane;
          const float xs = xr < a.n ? __ldg(a.xscale + xr) : 0.0f;
#pragma unroll
          for (int jj = 0; jj < 32; ++jj) v[c][jj] = (v[c][jj] * __shfl_sync(kFullMask, xs, jj)) * qs;
        }
        // one compare per score: the columns at or above the heap's minimum
        uint32_t mask = 0;
#pragma unroll
        for (int jj = 0; jj < 32; ++jj)
          mask |= ((c * 32 + jj < nvalid) && (hn < RS || v[c][jj] >= thr)) ? (1u << jj) : 0u;
        if (!live) mask = 0;
        if (__any_sync(kFullMask, mask != 0)) {
          // candidates: every lane takes its own next one per round, so the
          // warp runs as many rounds as its busiest lane has candidates
          float st[32];
#pragma unroll
          for (int jj = 0; jj < 32; ++jj) st[jj] = v[c][jj];
          while (__any_sync(kFullMask, mask != 0)) {
            if (mask) {
              const int jj = __ffs(mask) - 1;
              mask &= mask - 1;
              const float sc = st[jj];
              if (hn < RS || sc >= thr) {
                const unsigned long long key =
                    ((unsigned long long)ord_key(sc) << 32) | (uint32_t)~(uint32_t)(x0 + c * 32 + jj);
                key_heap_offer_strided(hk, kTile, hn, RS, key);
                if (hn == RS) thr = __uint_as_float(ord_key_inv_dev((uint32_t)(hk[0] >> 32)));
              }
            }
          }
        }
      }
    }
    if (live) {
      unsigned long long* out = a.heap + ((size_t)q * a.splits + split) * RS;
      for (int t = 0; t < hn; ++t) out[t] = hk[t * kTile];
      a.heap_n[(size_t)q * a.splits + split] = hn;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0 && s_abort) atomicOr(a.status, 1u);
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
  }
}

// ---------------------------------------------------------------- merge + exact re-score
constexpr int kMergeThreads = 256;
constexpr int kMergeMax = 4096;  // splits * R candidates per query

__device__ __forceinline__ float dot_canonical_rows(const float* q, const float* row, int nchunk, int lane) {
  float acc = 0.0f;
  const float4* r4 = reinterpret_cast<const float4*>(row);
  const float4* q4 = reinterpret_cast<const float4*>(q);
  for (int c = lane; c < nchunk; c += 32) {
    const float4 x = __ldg(r4 + c);
    const float4 y = q4[c];
    acc = fmaf(y.x, x.x, acc);
    acc = fmaf(y.y, x.y, acc);
    acc = fmaf(y.z, x.z, acc);
    acc = fmaf(y.w, x.w, acc);
  }
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) acc = __fadd_rn(acc, __shfl_xor_sync(kFullMask, acc, o));
  return acc;
}

__global__ void __launch_bounds__(kMergeThreads) k_bf_merge(const float* __restrict__ Q, int nq, int d,
                                                            const float* __restrict__ Xc, int ld,
                                                            const unsigned long long* __restrict__ heap,
                                                            const int* __restrict__ heap_n, int splits, int RS, int R,
                                                            int k,
                                                            int32_t* __restrict__ out, float* __restrict__ out_v) {
  __shared__ unsigned long long key[kMergeMax];
  __shared__ __align__(16) float qv[1024];
  __shared__ float esc[kMaxR];
  __shared__ int eid[kMaxR];
  __shared__ unsigned s_n;
  const int q = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_n = 0;
  const int nchunk = (d + 3) / 4;
  for (int i = tid; i < 4 * nchunk; i += kMergeThreads) qv[i] = i < d ? Q[(size_t)q * d + i] : 0.0f;
  __syncthreads();
  // candidates of every split, complemented keys: ascending = best first
  // (score desc, then id asc)
  for (int s = 0; s < splits; ++s) {
    const int cnt = heap_n[(size_t)q * splits + s];
    const size_t base = ((size_t)q * splits + s) * RS;
    for (int i = tid; i < cnt; i += kMergeThreads) {
      const unsigned pos = atomicAdd(&s_n, 1u);
      key[pos] = ~heap[base + i];
    }
  }
  __syncthreads();
  const int n = (int)s_n;
  int N = 1;
  while (N < n) N <<= 1;
  for (int i = n + tid; i < N; i += kMergeThreads) key[i] = ~0ull;
  __syncthreads();
  for (int k2 = 2; k2 <= N; k2 <<= 1)
    for (int j = k2 >> 1; j > 0; j >>= 1) {
      for (int t = tid; t < N; t += kMergeThreads) {
        const int p = t ^ j;
        if (p > t) {
          const unsigned long long x = key[t], y = key[p];
          const bool up = (t & k2) == 0;
          if ((x > y) == up) {
            key[t] = y;
            key[p] = x;
          }
        }
      }
      __syncthreads();
    }
  // exact FP32 re-score of the best R
  const int nr = min(n, R);
  for (int r = warp; r < nr; r += kMergeThreads / 32) {
    const int id = (int)(uint32_t)key[r];  // ~key's low half is ~~id
    const float sc = dot_canonical_rows(qv, Xc + (size_t)id * ld, nchunk, lane);
    if (lane == 0) {
      esc[r] = sc;
      eid[r] = id;
    }
  }
  __syncthreads();
  // top k by (score desc, id asc): rank by counting
  for (int r = tid; r < nr; r += kMergeThreads) {
    const uint32_t kr = ord_key(esc[r]);
    int rank = 0;
    for (int j = 0; j < nr; ++j) {
      const uint32_t kj = ord_key(esc[j]);
      rank += (kj > kr) || (kj == kr && eid[j] < eid[r]);
    }
    if (rank < k) {
      out[(size_t)q * k + rank] = eid[r];
      if (out_v) out_v[(size_t)q * k + rank] = esc[r];
    }
  }
  for (int j = nr + tid; j < k; j += kMergeThreads) {
    out[(size_t)q * k + j] = 0;
    if (out_v) out_v[(size_t)q * k + j] = 0.0f;
  }
}

// queries -> BF16 rows (ldo elements) or E4M3 rows with a per-query scale
__global__ void k_bf_queries(const float* __restrict__ Q, int nq, int d, int ldo, int mode, void* __restrict__ out,
                             float* __restrict__ qscale) {
  const int q = blockIdx.x;
  const int lane = threadIdx.x;  // one warp per query
  if (q >= nq) return;
  const float* qv = Q + (size_t)q * d;
  if (mode == kRowsBF16) {
    uint16_t* o = static_cast<uint16_t*>(out) + (size_t)q * ldo;
    for (int j = lane; j < ldo; j += 32) {
      const __nv_bfloat16 b = __float2bfloat16_rn(j < d ? qv[j] : 0.0f);
      o[j] = *reinterpret_cast<const uint16_t*>(&b);
    }
  } else {
    float mx = 0.0f;
    for (int j = lane; j < d; j += 32) mx = fmaxf(mx, fabsf(qv[j]));
    for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(kFullMask, mx, o));
    const float s = mx > 0.0f ? mx / 448.0f : 1.0f;
    uint8_t* o = static_cast<uint8_t*>(out) + (size_t)q * ldo;
    for (int j = lane; j < ldo; j += 32)
      o[j] = (uint8_t)__nv_cvt_float_to_fp8(j < d ? qv[j] / s : 0.0f, __NV_SATFINITE, __NV_E4M3);
    if (lane == 0) qscale[q] = s;
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult qr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &qr) == cudaSuccess &&
        qr == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// 2D map over rows of `row_bytes` (multiple of 16), `inner` valid bytes per
// row, boxes of 128 bytes x 128 rows, 128-byte swizzle, zero fill outside.
bool make_map(CUtensorMap* m, const void* base, long long rows, int inner_elems, int row_bytes, int esize) {
  auto enc = encode_fn();
  if (!enc) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)inner_elems, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)row_bytes};
  const cuuint32_t box[2] = {(cuuint32_t)(kBoxBytes / esize), (cuuint32_t)kTile};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r =
      enc(m, esize == 2 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base),
          dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <typename T>
cudaError_t grow(T*& p, size_t& cap, size_t need) {
  if (p && cap >= need) return cudaSuccess;
  cudaFree(p);
  p = nullptr;
  cap = 0;
  const cudaError_t e = dev_malloc(&p, std::max<size_t>(need, 1) * sizeof(T));
  if (e == cudaSuccess) cap = std::max<size_t>(need, 1);
  return e;
}

}  // namespace

void BfWorkspace::release() {
  cudaFree(qrows);
  cudaFree(qscale);
  cudaFree(heap);
  cudaFree(heap_n);
  cudaFree(status);
  *this = BfWorkspace();
}

}  // namespace fpp

extern "C" int fpp_bruteforce_topk_lowp(fpp_index* h, const float* d_queries, int n_queries, int n_neighbors,
                                        int precision, int shortlist_mult, int32_t* d_out, float* d_out_val,
                                        void* stream) {
  using namespace fpp;
  if (!h) return set_last_error(FPP_ERR_INVALID_ARGUMENT, "bruteforce_lowp: NULL handle");
  std::lock_guard<std::mutex> g(h->mu);
  if (!h->built) return set_last_error(FPP_ERR_NOT_BUILT, "bruteforce_lowp: the index is not built");
  if (precision != kRowsBF16 && precision != kRowsFP8)
    return set_last_error(FPP_ERR_INVALID_ARGUMENT, "bruteforce_lowp: precision must be 1 (BF16) or 2 (FP8)");
  const long long R = (long long)n_neighbors * shortlist_mult;
  if (n_neighbors < 1 || shortlist_mult < 1 || R > kMaxR)
    return set_last_error(FPP_ERR_INVALID_ARGUMENT, "bruteforce_lowp: need 1 <= k and k * shortlist_mult <= 256");
  if (n_queries < 0) return set_last_error(FPP_ERR_INVALID_ARGUMENT, "bruteforce_lowp: n_queries must be >= 0");
  if (n_queries == 0) return clear_last_error();
  if (!d_queries || !d_out) return set_last_error(FPP_ERR_INVALID_ARGUMENT, "bruteforce_lowp: NULL buffer");
  const int d = h->P.n_features;
  const int esize = precision == kRowsBF16 ? 2 : 1;
  if (d * esize > kKPadBytes || d > 1024)
    return set_last_error(FPP_ERR_UNSUPPORTED, "bruteforce_lowp: n_features * element size must be <= 512 bytes");
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return set_last_error(FPP_ERR_CUDA, std::string("bruteforce_lowp: ") + cudaGetErrorString(e));
  cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
  Error err{0, ""};
  int rc = ensure_lowp_rows(h->P, h->di, precision, s, err);
  if (rc) return set_last_error(rc, err.msg);
  BfWorkspace& scr = h->bfw;
  const int ldo = h->di.ld_lp;  // elements per stored row (BF16: d rounded to 8; E4M3: to 16)
  const int row_bytes = ldo * esize;
  const long long n = h->P.n_points;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
  const int qtiles = (n_queries + kTile - 1) / kTile;
  // splits of the rows: the choice whose waves of one CTA per SM come out
  // fullest (each split keeps its own shortlist heap per query)
  const long long xtiles = (n + kTile - 1) / kTile;
  const long long RS = std::min<long long>(R, kMaxRS);
  const long long max_splits = std::min<long long>({256, xtiles, kMergeMax / RS});
  // at least R / RS splits, so the splits' heaps hold R candidates together
  const long long min_splits = std::min<long long>(max_splits, (R + RS - 1) / RS);
  int splits = (int)min_splits;
  double best = -1.0;
  for (int sp = (int)min_splits; sp <= max_splits; ++sp) {
    const long long ctas = (long long)qtiles * sp;
    const double waves = (double)((ctas + nsm - 1) / nsm);
    const double eff = (double)ctas / (waves * nsm);
    if (eff > best + 1e-9) {
      best = eff;
      splits = sp;
    }
    if (ctas >= 8LL * nsm) break;
  }
  const long long rows_per_split = ((xtiles + splits - 1) / splits) * kTile;
  const size_t nheap = (size_t)n_queries * splits * (size_t)RS;
  if ((e = grow(scr.qrows, scr.cap_q, (size_t)qtiles * kTile * row_bytes)) ||
      (e = grow(scr.qscale, scr.cap_qs, (size_t)qtiles * kTile)) || (e = grow(scr.heap, scr.cap_hv, nheap)) ||
      (e = grow(scr.heap_n, scr.cap_n, (size_t)n_queries * splits)) ||
      (!scr.status && (e = dev_malloc(&scr.status, sizeof(unsigned)))))
    return set_last_error(e == cudaErrorMemoryAllocation ? FPP_ERR_OUT_OF_MEMORY : FPP_ERR_CUDA,
                          std::string("bruteforce_lowp: ") + cudaGetErrorString(e));
  k_bf_queries<<<n_queries, 32, 0, s>>>(d_queries, n_queries, d, ldo, precision, scr.qrows, scr.qscale);
  CUtensorMap qmap, xmap;
  if (!make_map(&qmap, scr.qrows, (long long)n_queries, ldo, row_bytes, esize) ||
      !make_map(&xmap, h->di.Xlp, n, ldo, row_bytes, esize))
    return set_last_error(FPP_ERR_CUDA, "bruteforce_lowp: cuTensorMapEncodeTiled failed");
  BfArgs a;
  a.n = (int)n;
  a.nq = n_queries;
  a.d = d;
  a.kbytes = ((d * esize + 31) / 32) * 32;
  a.boxes = (a.kbytes + kBoxBytes - 1) / kBoxBytes;
  a.stages = a.boxes <= 2 ? 4 : 2;  // 160 KB (32 KB tiles) or at most 192 KB of shared memory
  a.rows_per_split = (int)rows_per_split;
  a.splits = splits;
  a.qtiles = qtiles;
  a.R = (int)R;
  a.rs = (int)RS;
  a.xscale = h->di.Xlp_scale;
  a.qscale = scr.qscale;
  a.heap = scr.heap;
  a.heap_n = scr.heap_n;
  a.status = scr.status;
  const size_t smem = 1024 + (size_t)(1 + a.stages) * a.boxes * kBoxTileBytes + (size_t)kTile * RS * 8 +
                     (2 * a.stages + 5) * 8 + 16;
  const void* kern = precision == kRowsBF16 ? reinterpret_cast<const void*>(&k_bf_lowp<kRowsBF16>)
                                            : reinterpret_cast<const void*>(&k_bf_lowp<kRowsFP8>);
  if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess)
    return set_last_error(FPP_ERR_CUDA, std::string("bruteforce_lowp: smem attribute: ") + cudaGetErrorString(e));
  cudaMemsetAsync(scr.status, 0, sizeof(unsigned), s);
  void* args[] = {&qmap, &xmap, &a};
  if ((e = cudaLaunchKernel(kern, dim3((unsigned)(qtiles * splits)), dim3(kThreads), args, smem, s)) != cudaSuccess)
    return set_last_error(FPP_ERR_CUDA, std::string("bruteforce_lowp: launch: ") + cudaGetErrorString(e));
  k_bf_merge<<<n_queries, kMergeThreads, 0, s>>>(d_queries, n_queries, d, h->di.Xc, h->di.ld, scr.heap, scr.heap_n, splits, (int)RS, (int)R, n_neighbors, d_out, d_out_val);
  unsigned st = 0;
  e = cudaMemcpyAsync(&st, scr.status, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return set_last_error(FPP_ERR_CUDA, std::string("bruteforce_lowp: ") + cudaGetErrorString(e));
  if (st) return set_last_error(FPP_ERR_DEVICE, "bruteforce_lowp: a block gave up waiting on its pipeline");
  return clear_last_error();
}
