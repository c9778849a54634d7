// fpp_noalloc.cu — fpp_rerank_probes_noalloc: the gather / deduplicate /
// rerank / top-k stage of a query for callers that cannot allocate device
// memory.
//
// Who needs it: code that runs where cudaMalloc is off limits — a serving
// thread with a hard latency budget (cudaMalloc and cudaFree synchronise the
// device and can stall for milliseconds), or a host process whose device
// memory is owned by another allocator (a framework's caching pool, a
// pre-sized arena) that must not see foreign allocations.  fpp_query
// allocates its workspace on first use and grows it with the batch; this
// entry point allocates nothing.  The call waits for its kernel (it reads a
// status word back), so it is a blocking call on its stream.
//
// How: the per-block scratch the stage needs (a dedupe bitset of n bits, the
// unique-candidate list and its scores) lives in one file-scope __device__
// array of kScratchBytes (64 MiB).  Every GPU that loads the library holds that
// array until the process exits.  Host code cannot use the array's name as a
// device address, so the first call on each device looks the address up with
// cudaGetSymbolAddress (with that device current) and caches it.  Every call
// shares the one array and keeps the previous call's contents, so each call
// clears the status word and the bitsets of the blocks it uses before its
// kernel runs (the unique lists and scores are written before they are read);
// two calls whose kernels overlap on the GPU (two streams, or two handles on
// one device) race on it.
//
// The probes come from the caller, so every probe id is checked against the
// index's bucket count on the device: an id outside [0, n_tables * 4 *
// n_proj^2) reads nothing, sets a status bit, and the call returns
// FPP_ERR_INVALID_ARGUMENT.
//
// The results are those of fpp_query for the same probes: same canonical FP32
// dot order, same top-k with the exact heap replay on ties
// (src/FalconnPP.cpp:633-673).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/falconnpp_b200.h"
#include "fpp_device.cuh"
#include "fpp_handle.h"

namespace fpp {
namespace {

constexpr size_t kScratchBytes = 64ull << 20;  // the stated maximum
constexpr size_t kStatusBytes = 256;            // status word, padded to keep blocks aligned
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kProbeChunk = 2048;
constexpr int kMaxK = 1024;
constexpr int kMaxChunksPerLane = 8;
constexpr long long kTargetCap = 65536;  // unique candidates per query a block can hold
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_addr_mu;
unsigned char* g_addr[kMaxDevices] = {};

__host__ __device__ inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

struct NoAllocArgs {
  const uint32_t* probes;
  uint32_t nbuckets;  // n_tables * 4 * n_proj^2: valid probe ids are below it
  int nq, qProbes, k;
  const uint32_t* bucket_off;
  const int32_t* ids;
  const float* Xc;
  int ld;
  const float* Q;
  int d;
  long long nwords;
  long long cap;
  size_t block_bytes;
  unsigned char* scratch;  // device address of g_noalloc_scratch
  int32_t* out;
};

__device__ __forceinline__ float dot_canonical_dev(const float4* qc, int nchunk, const float* row, int lane) {
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

__global__ void __launch_bounds__(kThreads) k_gather_rerank_noalloc(NoAllocArgs a) {
  __shared__ uint32_t s_po[kProbeChunk];
  __shared__ uint32_t s_ps[kProbeChunk];
  __shared__ uint32_t hist[256];
  __shared__ unsigned s_u, s_ge, s_sel;
  __shared__ uint32_t s_prefix, s_remaining;
  __shared__ unsigned long long s_top[kMaxK];
  __shared__ float s_hv[kMaxK];
  __shared__ int s_hi[kMaxK];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  unsigned int* status = reinterpret_cast<unsigned int*>(a.scratch);
  unsigned char* mine = a.scratch + kStatusBytes + (size_t)blockIdx.x * a.block_bytes;
  uint32_t* bits = reinterpret_cast<uint32_t*>(mine);
  uint32_t* uq = reinterpret_cast<uint32_t*>(mine + align256((size_t)a.nwords * 4));
  uint32_t* sc = uq + align256((size_t)a.cap * 4) / 4;
  const int nchunk = (a.d + 3) / 4;
  const int k = a.k;
  const unsigned cap = (unsigned)a.cap;

  for (int q = blockIdx.x; q < a.nq; q += gridDim.x) {
    if (tid == 0) s_u = 0;
    __syncthreads();
    const uint32_t* pr = a.probes + (size_t)q * a.qProbes;
    for (int p0 = 0; p0 < a.qProbes; p0 += kProbeChunk) {
      const int np = min(kProbeChunk, a.qProbes - p0);
      for (int i = tid; i < np; i += kThreads) {
        const uint32_t g = pr[p0 + i];
        uint32_t o = 0, sz = 0;
        if (g < a.nbuckets) {
          o = a.bucket_off[g];
          sz = a.bucket_off[g + 1] - o;
        } else {
          atomicOr(status, 2u);  // a probe id outside the index: read nothing
        }
        s_po[i] = o;
        s_ps[i] = sz;
      }
      __syncthreads();
      for (int p = warp; p < np; p += kWarps) {
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
            const unsigned pos = base + __popc(bal & ((1u << lane) - 1u));
            if (fresh && pos < cap) uq[pos] = id;  // beyond cap: counted, not stored
          }
        }
      }
      __syncthreads();
    }
    const unsigned U = s_u;
    int32_t* orow = a.out + (size_t)q * k;
    if (U > cap) {
      // more unique candidates than this block can hold: report, zero the
      // row, and clear the whole bitset (not every set bit was recorded)
      if (tid == 0) atomicOr(status, 1u);
      for (int j = tid; j < k; j += kThreads) orow[j] = 0;
      for (long long w = tid; w < a.nwords; w += kThreads) bits[w] = 0u;
      __syncthreads();
      continue;
    }
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
      for (unsigned r = warp; r < U; r += kWarps) {
        const uint32_t id = uq[r];
        const float s = dot_canonical_dev(qc, nchunk, a.Xc + (size_t)id * a.ld, lane);
        if (lane == 0) sc[r] = __float_as_uint(s);
      }
    }
    __syncthreads();
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
        for (unsigned i = tid; i < U; i += kThreads) {
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
      if (tid == 0) s_ge = 0;
      __syncthreads();
      unsigned ge = 0;
      for (unsigned i = tid; i < U; i += kThreads) ge += ord_key_bits(sc[i]) >= t;
      atomicAdd(&s_ge, ge);
      __syncthreads();
      exact = (s_ge == kk);
      nsel = kk;
    }
    if (exact) {
      if (tid == 0) s_sel = 0;
      __syncthreads();
      for (unsigned i = tid; i < U; i += kThreads) {
        const uint32_t key = ord_key_bits(sc[i]);
        if (U <= kk || key >= t) {
          const unsigned pos = atomicAdd(&s_sel, 1u);
          s_top[pos] = ((unsigned long long)(~key) << 32) | uq[i];
        }
      }
      __syncthreads();
      int N = 1;
      while (N < (int)nsel) N <<= 1;
      for (int kk2 = 2; kk2 <= N; kk2 <<= 1) {
        for (int j = kk2 >> 1; j > 0; j >>= 1) {
          for (int tt = tid; tt < N / 2; tt += kThreads) {
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
      unsigned dup = 0;
      for (unsigned i = tid; i + 1 < nsel; i += kThreads) dup |= (s_top[i] >> 32) == (s_top[i + 1] >> 32);
      exact = !__syncthreads_or(dup);
    }
    if (exact) {
      for (int j = tid; j < k; j += kThreads) orow[j] = (unsigned)j < nsel ? (int32_t)(uint32_t)s_top[j] : 0;
    } else {
      block_bitonic_sort_u32(uq, sc, (int)U);
      if (tid == 0) {
        int n = 0;
        for (unsigned i = 0; i < U; ++i) topp_offer<int>(s_hv, s_hi, n, k, __uint_as_float(sc[i]), (int)uq[i]);
        for (int j = n; j < k; ++j) orow[j] = 0;
        for (int j = n - 1; j >= 0; --j) {
          orow[j] = s_hi[0];
          heap_pop<true, int>(s_hv, s_hi, n);
        }
      }
    }
    __syncthreads();
    for (unsigned i = tid; i < U; i += kThreads) bits[uq[i] >> 5] = 0u;
    __syncthreads();
  }
}

// Device address of the scratch array for the current device, looked up once
// per device (the first call on a device does it; do that before any capture).
int scratch_address(int dev, unsigned char** out) {
  if (dev < 0 || dev >= kMaxDevices) return set_last_error(FPP_ERR_DEVICE, "rerank_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> g(g_addr_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      return set_last_error(FPP_ERR_CUDA, std::string("rerank_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_addr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_addr[dev];
  return FPP_OK;
}

}  // namespace
}  // namespace fpp

extern "C" int fpp_rerank_probes_noalloc(fpp_index* h, const float* d_queries, int n_queries,
                                         const uint32_t* d_probes, int n_probes, int n_neighbors,
                                         int32_t* d_out, void* stream) {
  using namespace fpp;
  if (!h) return set_last_error(FPP_ERR_INVALID_ARGUMENT, "rerank_noalloc: NULL handle");
  std::lock_guard<std::mutex> g(h->mu);
  if (!h->built) return set_last_error(FPP_ERR_NOT_BUILT, "rerank_noalloc: the index is not built");
  if (n_queries < 0 || n_probes < 1) return set_last_error(FPP_ERR_INVALID_ARGUMENT, "rerank_noalloc: bad sizes");
  if (n_neighbors < 1 || n_neighbors > kMaxK)
    return set_last_error(FPP_ERR_INVALID_ARGUMENT, "rerank_noalloc: n_neighbors must be in [1, 1024]");
  if (n_queries == 0) return clear_last_error();
  if (!d_queries || !d_probes || !d_out) return set_last_error(FPP_ERR_INVALID_ARGUMENT, "rerank_noalloc: NULL buffer");
  if (h->P.n_features > 32 * 4 * kMaxChunksPerLane)
    return set_last_error(FPP_ERR_UNSUPPORTED, "rerank_noalloc: n_features must be <= 1024");
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return set_last_error(FPP_ERR_CUDA, std::string("rerank_noalloc: ") + cudaGetErrorString(e));
  unsigned char* scratch = nullptr;
  int rc = scratch_address(h->device, &scratch);
  if (rc) return rc;

  // per-block layout: bitset (n bits) | unique ids (cap) | scores (cap)
  const long long nwords = ((long long)h->P.n_points + 31) / 32;
  const size_t bitset_bytes = align256((size_t)nwords * 4);
  const size_t avail = kScratchBytes - kStatusBytes;
  if (bitset_bytes + 2 * align256((size_t)n_neighbors * 4) > avail)
    return set_last_error(FPP_ERR_UNSUPPORTED,
                          "rerank_noalloc: n_points too large for the 64 MiB scratch (limit about 500M points)");
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
  long long cap = kTargetCap;
  const size_t per_block_target = bitset_bytes + 2 * align256((size_t)cap * 4);
  long long grid = std::min<long long>({(long long)n_queries, (long long)nsm, (long long)(avail / per_block_target)});
  if (grid < 1) {  // one block: give it everything that is left
    grid = 1;
    cap = (long long)((avail - bitset_bytes) / 2 / 256 * 256 / 4);
  }
  const size_t block_bytes = bitset_bytes + 2 * align256((size_t)cap * 4);
  cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
  // what must start at zero: the status word and the bitsets of the blocks
  // used (one row of bitset_bytes at the start of each block's region)
  e = cudaMemsetAsync(scratch, 0, kStatusBytes, s);
  if (e == cudaSuccess) e = cudaMemset2DAsync(scratch + kStatusBytes, block_bytes, 0, bitset_bytes, (size_t)grid, s);
  if (e != cudaSuccess) return set_last_error(FPP_ERR_CUDA, std::string("rerank_noalloc: memset: ") + cudaGetErrorString(e));
  NoAllocArgs a;
  a.probes = d_probes;
  a.nbuckets = (uint32_t)((long long)h->P.n_tables * 4LL * h->P.n_proj * h->P.n_proj);
  a.nq = n_queries;
  a.qProbes = n_probes;
  a.k = n_neighbors;
  a.bucket_off = h->di.bucket_off;
  a.ids = h->di.ids;
  a.Xc = h->di.Xc;
  a.ld = h->di.ld;
  a.Q = d_queries;
  a.d = h->P.n_features;
  a.nwords = nwords;
  a.cap = cap;
  a.block_bytes = block_bytes;
  a.scratch = scratch;
  a.out = d_out;
  k_gather_rerank_noalloc<<<(unsigned)grid, kThreads, 0, s>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_last_error(FPP_ERR_CUDA, std::string("rerank_noalloc: launch: ") + cudaGetErrorString(e));
  unsigned int status = 0;
  e = cudaMemcpyAsync(&status, scratch, sizeof(status), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return set_last_error(FPP_ERR_CUDA, std::string("rerank_noalloc: ") + cudaGetErrorString(e));
  if (status & 2u)
    return set_last_error(FPP_ERR_INVALID_ARGUMENT,
                          "rerank_noalloc: a probe id is outside [0, n_tables * 4 * n_proj^2); it was read as an "
                          "empty bucket");
  if (status)
    return set_last_error(FPP_ERR_UNSUPPORTED,
                          "rerank_noalloc: a query has more unique candidates than the scratch holds per block "
                          "(65536 when n_points allows); its row was zeroed — use fpp_query for it");
  return clear_last_error();
}
