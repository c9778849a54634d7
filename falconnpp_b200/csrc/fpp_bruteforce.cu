// fpp_bruteforce.cu — exact maximum-inner-product top-k in FP64 on the GPU
// (model: BF::mips_topK, src/BF.cpp:17-86), the ground truth the recall of the
// index is measured against.  Ties are broken by ascending id.
//
//   k_bf_partial: a block takes QB = 8 queries and a slice of the points; each
//                 thread scores one point against the 8 queries (FP32 inputs
//                 widened to FP64, FP64 fma), and per query the block keeps the
//                 best k of its slice in shared memory: candidates above the
//                 running k-th score are appended to a buffer that is sorted
//                 and cut back to k when it fills;
//   k_bf_merge:   one block per query merges the slices' best-k lists.
// FP64 is used only here.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <string>

#include "../../include/falconnpp_b200.h"
#include "fpp_handle.h"

namespace fpp {
namespace {

constexpr int kQB = 8;         // queries per block
constexpr int kBfThreads = 256;
constexpr int kBfMaxK = 256;
constexpr int kCap = 1024;     // candidate buffer per query (>= k + kBfThreads)

// order-preserving key of a double: larger value -> larger key
__device__ __forceinline__ unsigned long long dkey(double v) {
  unsigned long long u = (unsigned long long)__double_as_longlong(v);
  if ((u << 1) == 0ull) return 0x8000000000000000ull;  // -0 == +0
  return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}

// a before b: larger key, then smaller id
__device__ __forceinline__ bool before(unsigned long long ka, uint32_t ia, unsigned long long kb, uint32_t ib) {
  return ka > kb || (ka == kb && ia < ib);
}

// sort n (key, id) pairs so that entry 0 is the best (bitonic, all comparators
// in the same direction; positions >= n never move)
__device__ void block_sort_pairs(unsigned long long* key, uint32_t* id, int n) {
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
        if (hi < n && before(key[hi], id[hi], key[lo], id[lo])) {
          const unsigned long long tk = key[lo];
          key[lo] = key[hi];
          key[hi] = tk;
          const uint32_t ti = id[lo];
          id[lo] = id[hi];
          id[hi] = ti;
        }
      }
      __syncthreads();
    }
}

struct BfArgs {
  const float* X;  // n x d
  long long n;
  int d;
  const float* Q;  // nq x d
  int nq, k;
  long long per_slice;
  unsigned long long* pkey;  // [nq][slices][k]
  uint32_t* pid;
  int slices;
};

__global__ void __launch_bounds__(kBfThreads) k_bf_partial(BfArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  double* qs = reinterpret_cast<double*>(smem);                                  // kQB x d
  unsigned long long* ck = reinterpret_cast<unsigned long long*>(qs + (size_t)kQB * a.d);  // kQB x kCap
  uint32_t* ci = reinterpret_cast<uint32_t*>(ck + (size_t)kQB * kCap);          // kQB x kCap
  __shared__ unsigned cnt[kQB];
  __shared__ unsigned long long thr[kQB];
  __shared__ int need_sort;
  const int q0 = blockIdx.x * kQB;
  const int slice = blockIdx.y;
  const long long p0 = (long long)slice * a.per_slice;
  const long long p1 = min(a.n, p0 + a.per_slice);
  for (int i = threadIdx.x; i < kQB * a.d; i += kBfThreads) {
    const int b = i / a.d;
    qs[i] = (q0 + b < a.nq) ? (double)a.Q[(size_t)(q0 + b) * a.d + (i - b * a.d)] : 0.0;
  }
  if (threadIdx.x < kQB) {
    cnt[threadIdx.x] = 0;
    thr[threadIdx.x] = 0ull;  // below every real key: accept everything until k are held
  }
  __syncthreads();
  for (long long base = p0; base < p1; base += kBfThreads) {
    const long long p = base + threadIdx.x;
    double s[kQB];
#pragma unroll
    for (int b = 0; b < kQB; ++b) s[b] = 0.0;
    if (p < p1) {
      const float* x = a.X + (size_t)p * a.d;
      for (int j = 0; j < a.d; ++j) {
        const double xv = (double)__ldg(x + j);
#pragma unroll
        for (int b = 0; b < kQB; ++b) s[b] = fma(qs[b * a.d + j], xv, s[b]);
      }
    }
#pragma unroll
    for (int b = 0; b < kQB; ++b) {
      if (p < p1 && q0 + b < a.nq) {
        const unsigned long long key = dkey(s[b]);
        if (key >= thr[b]) {
          const unsigned pos = atomicAdd(&cnt[b], 1u);
          ck[b * kCap + pos] = key;  // pos < kCap: the buffer is cut back before it can fill
          ci[b * kCap + pos] = (uint32_t)p;
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int ns = 0;
      for (int b = 0; b < kQB; ++b) ns |= (cnt[b] + kBfThreads > kCap) ? (1 << b) : 0;
      need_sort = ns;
    }
    __syncthreads();
    const int ns = need_sort;
    for (int b = 0; b < kQB; ++b) {
      if (!((ns >> b) & 1)) continue;
      block_sort_pairs(ck + b * kCap, ci + b * kCap, (int)cnt[b]);
      if (threadIdx.x == 0) {
        cnt[b] = min(cnt[b], (unsigned)a.k);
        thr[b] = ck[b * kCap + a.k - 1];
      }
      __syncthreads();
    }
  }
  for (int b = 0; b < kQB; ++b) {
    if (q0 + b >= a.nq) break;
    block_sort_pairs(ck + b * kCap, ci + b * kCap, (int)cnt[b]);
    const unsigned c = cnt[b];
    for (int i = threadIdx.x; i < a.k; i += kBfThreads) {
      const size_t o = ((size_t)(q0 + b) * a.slices + slice) * a.k + i;
      a.pkey[o] = (unsigned)i < c ? ck[b * kCap + i] : 0ull;
      a.pid[o] = (unsigned)i < c ? ci[b * kCap + i] : 0xffffffffu;
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kBfThreads) k_bf_merge(const unsigned long long* pkey, const uint32_t* pid,
                                                          int slices, int k, int32_t* out, double* out_val) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int n = slices * k;
  unsigned long long* key = reinterpret_cast<unsigned long long*>(smem);
  uint32_t* id = reinterpret_cast<uint32_t*>(key + n);
  const int q = blockIdx.x;
  for (int i = threadIdx.x; i < n; i += kBfThreads) {
    key[i] = pkey[(size_t)q * n + i];
    id[i] = pid[(size_t)q * n + i];
  }
  __syncthreads();
  block_sort_pairs(key, id, n);
  for (int i = threadIdx.x; i < k; i += kBfThreads) {
    const bool real = id[i] != 0xffffffffu;
    out[(size_t)q * k + i] = real ? (int32_t)id[i] : -1;
    if (out_val) {
      unsigned long long u = key[i];
      u = (u & 0x8000000000000000ull) ? (u ^ 0x8000000000000000ull) : ~u;
      out_val[(size_t)q * k + i] = real ? __longlong_as_double((long long)u) : 0.0;
    }
  }
}

}  // namespace
}  // namespace fpp

extern "C" int fpp_bruteforce_topk_f64(const float* d_X, long long n_points, int n_features, const float* d_Q,
                                       int n_queries, int k, int32_t* d_out, double* d_out_val, void* stream) {
  using namespace fpp;
  if (!d_X || !d_Q || !d_out || n_points < 1 || n_features < 1 || n_queries < 0)
    return set_last_error(FPP_ERR_INVALID_ARGUMENT, "bruteforce: NULL buffer or bad sizes");
  if (k < 1 || k > kBfMaxK || k > n_points)
    return set_last_error(FPP_ERR_INVALID_ARGUMENT, "bruteforce: need 1 <= k <= min(256, n_points)");
  if (n_features > 1024) return set_last_error(FPP_ERR_UNSUPPORTED, "bruteforce: n_features must be <= 1024");
  if (n_points >= (1LL << 32) - 1) return set_last_error(FPP_ERR_UNSUPPORTED, "bruteforce: too many points");
  if (n_queries == 0) return clear_last_error();
  cudaStream_t s = (cudaStream_t)stream;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int qblocks = (n_queries + kQB - 1) / kQB;
  // slices: enough blocks to fill the GPU, each at least a few thousand points
  long long slices = std::max(1LL, std::min<long long>((long long)nsm * 4 / qblocks + 1, n_points / 4096 + 1));
  slices = std::min<long long>(slices, 8192 / k);  // merge buffer fits in shared memory
  const long long per_slice = (n_points + slices - 1) / slices;
  unsigned long long* pkey = nullptr;
  uint32_t* pid = nullptr;
  const size_t np = (size_t)n_queries * slices * k;
  cudaError_t e = fpp::dev_malloc(&pkey, sizeof(unsigned long long) * np);
  if (e == cudaSuccess) e = fpp::dev_malloc(&pid, sizeof(uint32_t) * np);
  if (e != cudaSuccess) {
    cudaFree(pkey);
    return set_last_error(FPP_ERR_OUT_OF_MEMORY, "bruteforce: cannot allocate the partial lists");
  }
  BfArgs a;
  a.X = d_X;
  a.n = n_points;
  a.d = n_features;
  a.Q = d_Q;
  a.nq = n_queries;
  a.k = k;
  a.per_slice = per_slice;
  a.pkey = pkey;
  a.pid = pid;
  a.slices = (int)slices;
  const size_t smem1 = (size_t)kQB * n_features * 8 + (size_t)kQB * kCap * 12;
  const size_t smem2 = (size_t)slices * k * 12;
  cudaFuncSetAttribute(k_bf_partial, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem1);
  cudaFuncSetAttribute(k_bf_merge, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2);
  k_bf_partial<<<dim3(qblocks, (unsigned)slices), kBfThreads, smem1, s>>>(a);
  k_bf_merge<<<n_queries, kBfThreads, smem2, s>>>(pkey, pid, (int)slices, k, d_out, d_out_val);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(pkey);
  cudaFree(pid);
  if (e != cudaSuccess) return set_last_error(FPP_ERR_CUDA, std::string("bruteforce: ") + cudaGetErrorString(e));
  return clear_last_error();
}
