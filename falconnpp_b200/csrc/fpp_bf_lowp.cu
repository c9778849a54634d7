// fpp_bf_lowp.cu — brute-force maximum-inner-product search over the index's
// BF16 or FP8-E4M3 row copies on the tcgen05 tensor cores, with the top-R
// selection fused into the accumulator epilogue and an exact FP32 re-score of
// the shortlist (the block rerank of the precision form; model: BF::mips_topK,
// src/BF.cpp:17-86, an exact GEMV + size-k min-heap per query).
//
// k_bf_lowp — one persistent CTA per SM.  The (query tile of 128, row tile
// of 128) pairs, in query-tile-major order, are cut into units of equal
// length; CTA c takes units [c P, c P + P), a contiguous range, so every SM
// gets the same number of MMAs.  A segment is a unit's part inside one query
// tile; the query tile changes only between segments.
//   warp 0      TMA producer: the query tile at each change of query tile
//               (once the MMAs of the previous one have retired), row tiles
//               into a ring of shared-memory stages (128-byte swizzle, K-major);
//   warp 1      owns TMEM (256 columns: two 128-column accumulators) and
//               issues tcgen05.mma (M = 128 queries, N = 128 rows, K = 16
//               BF16 / 32 E4M3 per instruction, FP32 accumulate), committing
//               each tile to the stage's "empty" and the accumulator's "full"
//               barrier, and the last tile of a query tile to "query empty";
//   warps 2..5  epilogue: thread = one query (TMEM lane), reads its 128
//               scores with tcgen05.ld, applies the FP8 row scales (staged in
//               shared memory per tile), and keeps the segment's top RS keys
//               (score, ~id) in a shared-memory heap, so the kept set is the
//               segment's best by (score desc, id asc) even among equal
//               scores.  A chunk of 32 columns whose maximum is below every
//               lane's heap minimum is skipped after one max per score; the
//               others insert their candidates in warp-synchronous rounds.
//               At the end of a segment the heap goes to global memory.
// Long segments keep the heaps warm (few insertions), and the query tiles
// that read the same rows run side by side, so a row tile comes from HBM
// about once and from L2 for the others.
//
// k_bf_merge — one block per query: the segments' candidates, the best R by
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
constexpr int kMaxRS = 32;          // per-segment heap in shared memory: 128 queries x 32 keys = 32 KB
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
  int qtiles;
  long long xtiles;            // row tiles of 128
  long long tiles_per_unit;    // a unit: this many consecutive (query tile, row tile) tiles
  int units_per_cta;
  int max_segs;                // segments of one query tile, at most
  int R;                       // shortlist per query (merge)
  int rs;                      // per-segment heap size, min(R, kMaxRS)
  const float* xscale;         // FP8 per-row scales (nullable for BF16)
  unsigned long long* heap;    // [nq][max_segs][rs] keys (ord(score) << 32) | ~id
  int* heap_n;                 // [nq][max_segs] (zero for a segment that does not exist)
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

// The CTA's tiles: the contiguous range [c0, c1) of the (query tile, row
// tile) order t = qt * xtiles + xt, units_per_cta units of tiles_per_unit
// tiles.  A segment is the part of a unit inside one query tile; each keeps
// its own top-RS per query.
struct TileWalk {
  long long c0, T;
  int ntiles;
  __device__ TileWalk(const BfArgs& a) {
    T = (long long)a.qtiles * a.xtiles;
    const long long span = (long long)a.units_per_cta * a.tiles_per_unit;
    c0 = (long long)blockIdx.x * span;
    const long long c1 = min(T, c0 + span);
    ntiles = c1 > c0 ? (int)(c1 - c0) : 0;
  }
};

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
  float* xs_smem = reinterpret_cast<float*>(heap_smem + (size_t)kTile * a.rs);  // FP8: 4 x 128 row scales
  uint64_t* bars = reinterpret_cast<uint64_t*>(xs_smem + (MODE == kRowsFP8 ? 4 * kTile : 0));
  // bars: [0..S) full, [S..2S) empty, [2S, 2S+1] acc full, [2S+2, 2S+3] acc
  // empty, [2S+4] query tile full, [2S+5] query tile empty
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * a.stages + 6);
  __shared__ int s_abort;

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int S = a.stages;
  const TileWalk tw(a);
  const int ntiles = tw.ntiles;
  const long long xtiles = a.xtiles;
  const int ksteps = a.kbytes / 32;
  auto bar = [&](int i) { return smem_u32(bars + i); };
  const int B_FULL = 0, B_EMPTY = S, B_ACCF = 2 * S, B_ACCE = 2 * S + 2, B_QF = 2 * S + 4, B_QE = 2 * S + 5;
  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int s = 0; s < S; ++s) {
      mbar_init(bar(B_FULL + s), 1);
      mbar_init(bar(B_EMPTY + s), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(bar(B_ACCF + b), 1);
      mbar_init(bar(B_ACCE + b), 4);  // one arrival per epilogue warp
    }
    mbar_init(bar(B_QF), 1);
    mbar_init(bar(B_QE), 1);
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
    // ---- producer: a query tile at each change of query tile (once the
    // MMAs of the previous one are done), row tiles into the stage ring
    if (lane == 0) {
      int issued = 0, qloads = 0;
      bool ok = true;
      for (int i = 0; i < ntiles && ok; ++i) {
        const long long t = tw.c0 + i;
        const long long qt = t / xtiles;
        const long long xt = t - qt * xtiles;
        if (i == 0 || xt == 0) {
          if (qloads > 0) ok = mbar_wait(bar(B_QE), (qloads - 1) & 1, abort_flag);
          if (!ok) break;
          mbar_expect_tx(bar(B_QF), (uint32_t)tile_bytes);
          for (int bx = 0; bx < a.boxes; ++bx)
            tma_load_2d(smem_u32(q_smem + bx * kBoxTileBytes), &qmap, bx * C::box_elems, (int)(qt * kTile), bar(B_QF));
          ++qloads;
        }
        const int s = i % S;
        ok = mbar_wait(bar(B_EMPTY + s), ((i / S) & 1) ^ 1, abort_flag);
        if (!ok) break;
        mbar_expect_tx(bar(B_FULL + s), (uint32_t)tile_bytes);
        unsigned char* dst = x_smem + (size_t)s * tile_bytes;
        for (int bx = 0; bx < a.boxes; ++bx)
          tma_load_2d(smem_u32(dst + bx * kBoxTileBytes), &xmap, bx * C::box_elems, (int)(xt * kTile), bar(B_FULL + s));
        issued = i + 1;
      }
      // let every copy issued land before the CTA can exit (bounded)
      volatile int never = 0;
      if (qloads > 0) mbar_wait(bar(B_QF), (qloads - 1) & 1, &never);
      for (int i = max(0, issued - S); i < issued; ++i) mbar_wait(bar(B_FULL + i % S), (i / S) & 1, &never);
    }
  } else if (warp == 1) {
    // ---- MMA issuer
    if (lane == 0) {
      const uint32_t qa = smem_u32(q_smem);
      int issued = 0, qruns = 0;
      bool ok = true;
      for (int i = 0; i < ntiles && ok; ++i) {
        const long long t = tw.c0 + i;
        const long long xt = t % xtiles;
        if (i == 0 || xt == 0) {
          ok = mbar_wait(bar(B_QF), qruns & 1, abort_flag);
          if (!ok) break;
          ++qruns;
        }
        const int s = i % S;
        const int b = i & 1;
        ok = mbar_wait(bar(B_ACCE + b), ((i >> 1) & 1) ^ 1, abort_flag);
        if (!ok) break;
        ok = mbar_wait(bar(B_FULL + s), (i / S) & 1, abort_flag);
        if (!ok) break;
        tc_fence_after();
        const uint32_t xa = smem_u32(x_smem + (size_t)s * tile_bytes);
        for (int k = 0; k < ksteps; ++k) {
          const uint32_t off = (uint32_t)((k >> 2) * kBoxTileBytes + (k & 3) * 32);
          umma<MODE>(tmem + (uint32_t)(b * kTile), umma_desc_sw128(qa + off), umma_desc_sw128(xa + off),
                     k > 0 ? 1u : 0u);
        }
        umma_commit(bar(B_EMPTY + s));
        umma_commit(bar(B_ACCF + b));
        // the last tile of this query tile: its MMAs release the query tile
        if (i + 1 < ntiles && (t + 1) % xtiles == 0) umma_commit(bar(B_QE));
        issued = i + 1;
      }
      if (issued > 0) {  // the last tile's MMAs complete before TMEM is freed
        volatile int never = 0;
        mbar_wait(bar(B_ACCF + ((issued - 1) & 1)), ((issued - 1) >> 1) & 1, &never);
      }
    }
  } else {
    // ---- epilogue: thread = query of the tile (TMEM lane)
    const int quad = warp & 3;  // the TMEM lanes this warp may read
    const int ql = quad * 32 + lane;
    const int RS = a.rs;
    // the segment's top RS keys of this query in shared memory, slot j at
    // hk[j * kTile] (consecutive queries in consecutive words)
    unsigned long long* hk = heap_smem + ql;
    float* xs_w = xs_smem + (warp - 2) * kTile;  // FP8: this warp's copy of the tile's row scales
    int hn = 0;
    float thr = -INFINITY;  // score of the heap's minimum once the heap is full
    for (int i = 0; i < ntiles; ++i) {
      const long long t = tw.c0 + i;
      const long long qt = t / xtiles;
      const long long xt = t - qt * xtiles;
      const int q = (int)(qt * kTile) + ql;
      const bool live = q < a.nq;
      const int x0 = (int)(xt * kTile);
      const int nvalid = min(kTile, a.n - x0);
      const int b = i & 1;
      float4 xs4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      if (MODE == kRowsFP8) {  // this tile's scales, loaded before the wait
        const int xr = x0 + 4 * lane;
        if (xr + 3 < a.n) {
          xs4 = __ldg(reinterpret_cast<const float4*>(a.xscale + xr));
        } else {
          if (xr < a.n) xs4.x = __ldg(a.xscale + xr);
          if (xr + 1 < a.n) xs4.y = __ldg(a.xscale + xr + 1);
          if (xr + 2 < a.n) xs4.z = __ldg(a.xscale + xr + 2);
        }
      }
      // warp-uniform: the loads and votes below need every lane
      if (!__all_sync(kFullMask, mbar_wait(bar(B_ACCF + b), (i >> 1) & 1, abort_flag))) break;
      tc_fence_after();
      float v[4][32];
      const uint32_t taddr = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(b * kTile);
#pragma unroll
      for (int c = 0; c < 4; ++c) tmem_ld32(taddr + c * 32, v[c]);
      tmem_wait_ld();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(bar(B_ACCE + b));
      if (MODE == kRowsFP8) {
        reinterpret_cast<float4*>(xs_w)[lane] = xs4;
        __syncwarp();
      }
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        if (MODE == kRowsFP8) {
          // column j's row scale (the query's scale is one positive factor for
          // all of its keys, so it is left out of the ordering)
#pragma unroll
          for (int j4 = 0; j4 < 8; ++j4) {
            const float4 s4 = reinterpret_cast<const float4*>(xs_w)[c * 8 + j4];
            v[c][4 * j4] *= s4.x;
            v[c][4 * j4 + 1] *= s4.y;
            v[c][4 * j4 + 2] *= s4.z;
            v[c][4 * j4 + 3] *= s4.w;
          }
        }
        // the chunk's maximum: no column can enter a full heap below it
        float m0 = fmaxf(v[c][0], v[c][1]), m1 = fmaxf(v[c][2], v[c][3]);
        float m2 = fmaxf(v[c][4], v[c][5]), m3 = fmaxf(v[c][6], v[c][7]);
#pragma unroll
        for (int jj = 8; jj < 32; jj += 4) {
          m0 = fmaxf(m0, v[c][jj]);
          m1 = fmaxf(m1, v[c][jj + 1]);
          m2 = fmaxf(m2, v[c][jj + 2]);
          m3 = fmaxf(m3, v[c][jj + 3]);
        }
        const float m = fmaxf(fmaxf(m0, m1), fmaxf(m2, m3));
        const bool cand = live && (hn < RS || m >= thr);
        if (!__any_sync(kFullMask, cand)) continue;
        // candidates: the columns at or above the heap's minimum
        uint32_t mask = 0;
#pragma unroll
        for (int jj = 0; jj < 32; ++jj)
          mask |= ((c * 32 + jj < nvalid) && (hn < RS || v[c][jj] >= thr)) ? (1u << jj) : 0u;
        if (!cand) mask = 0;
        // every lane takes its own next candidate per round, so the warp runs
        // as many rounds as its busiest lane has candidates
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
      // the segment ends with this tile: its keys out, the heap emptied
      const bool seg_end = (i + 1 == ntiles) || ((t + 1) % xtiles == 0) || ((t + 1) % a.tiles_per_unit == 0);
      if (seg_end) {
        if (live) {
          const int seg = (int)(t / a.tiles_per_unit - (qt * xtiles) / a.tiles_per_unit);
          unsigned long long* out = a.heap + ((size_t)q * a.max_segs + seg) * RS;
          for (int j = 0; j < hn; ++j) out[j] = hk[j * kTile];
          a.heap_n[(size_t)q * a.max_segs + seg] = hn;
        }
        hn = 0;
        thr = -INFINITY;
      }
      if (MODE == kRowsFP8) __syncwarp();  // the scales are rewritten by the next tile
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
constexpr int kMergeMax = 4096;  // segments * RS candidates per query

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
                                                            const int* __restrict__ heap_n, int segs, int RS, int R,
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
  // candidates of every segment, complemented keys: ascending = best first
  // (score desc, then id asc)
  for (int s = 0; s < segs; ++s) {
    const int cnt = heap_n[(size_t)q * segs + s];
    const size_t base = ((size_t)q * segs + s) * RS;
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
  // one CTA per SM over the (query tile, row tile) order, in units of equal
  // length; each unit's part in one query tile (a segment) keeps its own
  // top-RS per query.  Units are at most xtiles / ceil(R / RS) tiles long, so
  // a query tile has at least ceil(R / RS) segments and R candidates fit.
  const long long xtiles = (n + kTile - 1) / kTile;
  const long long T = (long long)qtiles * xtiles;
  const long long RS = std::min<long long>(R, kMaxRS);
  const long long need = (R + RS - 1) / RS;
  const long long tu_max = std::max<long long>(1, xtiles / need);
  // P units per CTA, then the unit length that spreads the tiles over nsm x P
  // units: every SM gets the same work
  const long long per_cta = std::max<long long>(1, (T + (long long)nsm * tu_max - 1) / ((long long)nsm * tu_max));
  // few query tiles: units long enough that a query tile's segments fit the
  // merge (at most kMergeMax / RS, one more where a unit straddles two tiles)
  const long long seg_max = kMergeMax / RS - 1;
  const long long tu_merge = (xtiles + seg_max - 1) / seg_max;
  const long long tu = std::max<long long>(
      {1LL, tu_merge, (T + (long long)nsm * per_cta - 1) / ((long long)nsm * per_cta)});
  const long long units = (T + tu - 1) / tu;
  const long long grid = (units + per_cta - 1) / per_cta;
  const long long max_segs = (xtiles + tu - 1) / tu + 1;
  if (max_segs * RS > kMergeMax)
    return set_last_error(FPP_ERR_UNSUPPORTED, "bruteforce_lowp: too many row segments per query tile");
  const size_t nheap = (size_t)n_queries * max_segs * (size_t)RS;
  if ((e = grow(scr.qrows, scr.cap_q, (size_t)qtiles * kTile * row_bytes)) ||
      (e = grow(scr.qscale, scr.cap_qs, (size_t)qtiles * kTile)) || (e = grow(scr.heap, scr.cap_hv, nheap)) ||
      (e = grow(scr.heap_n, scr.cap_n, (size_t)n_queries * max_segs)) ||
      (!scr.status && (e = dev_malloc(&scr.status, sizeof(unsigned)))))
    return set_last_error(e == cudaErrorMemoryAllocation ? FPP_ERR_OUT_OF_MEMORY : FPP_ERR_CUDA,
                          std::string("bruteforce_lowp: ") + cudaGetErrorString(e));
  cudaMemsetAsync(scr.heap_n, 0, sizeof(int) * (size_t)n_queries * max_segs, s);
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
  a.qtiles = qtiles;
  a.xtiles = xtiles;
  a.tiles_per_unit = tu;
  a.units_per_cta = (int)per_cta;
  a.max_segs = (int)max_segs;
  a.R = (int)R;
  a.rs = (int)RS;
  a.xscale = h->di.Xlp_scale;
  a.heap = scr.heap;
  a.heap_n = scr.heap_n;
  a.status = scr.status;
  const size_t smem = 1024 + (size_t)(1 + a.stages) * a.boxes * kBoxTileBytes + (size_t)kTile * RS * 8 +
                     (precision == kRowsFP8 ? 4 * kTile * 4 : 0) + (2 * a.stages + 6) * 8 + 16;
  const void* kern = precision == kRowsBF16 ? reinterpret_cast<const void*>(&k_bf_lowp<kRowsBF16>)
                                            : reinterpret_cast<const void*>(&k_bf_lowp<kRowsFP8>);
  if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess)
    return set_last_error(FPP_ERR_CUDA, std::string("bruteforce_lowp: smem attribute: ") + cudaGetErrorString(e));
  cudaMemsetAsync(scr.status, 0, sizeof(unsigned), s);
  void* args[] = {&qmap, &xmap, &a};
  if ((e = cudaLaunchKernel(kern, dim3((unsigned)grid), dim3(kThreads), args, smem, s)) != cudaSuccess)
    return set_last_error(FPP_ERR_CUDA, std::string("bruteforce_lowp: launch: ") + cudaGetErrorString(e));
  k_bf_merge<<<n_queries, kMergeThreads, 0, s>>>(d_queries, n_queries, d, h->di.Xc, h->di.ld, scr.heap, scr.heap_n,
                                                 (int)max_segs, (int)RS, (int)R, n_neighbors, d_out, d_out_val);
  unsigned st = 0;
  e = cudaMemcpyAsync(&st, scr.status, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return set_last_error(FPP_ERR_CUDA, std::string("bruteforce_lowp: ") + cudaGetErrorString(e));
  if (st) return set_last_error(FPP_ERR_DEVICE, "bruteforce_lowp: a block gave up waiting on its pipeline");
  return clear_last_error();
}
