// fpp_batch_ext.cu — instances of the fused batched kernel that start from
// per-table probe lists computed by the exact FP32 hash kernel (kHashExt):
// probe cut, gather / dedupe, rerank and top-k only.  The fhtDim template
// argument only sizes shared-memory regions the hashing would use, so one
// value serves every index.
#include "fpp_batch_kernel.cuh"
#include "fpp_heap.h"

namespace fpp {

// ---------------------------------------------------------------- probe cut
// k_probe_cut — one block per query: the global top-qProbes of the query's
// L * m per-table lists (FalconnPP.cpp:540-582), ranked by counting exactly
// as the fused kernel's small-list cut does, with the reference's heap
// replayed when a tie straddles the cut; then the probed buckets' offsets and
// the inclusive prefix of their sizes.  The fused kernel starts its gather
// from these.
constexpr int kPcThreads = 128;

__global__ void __launch_bounds__(kPcThreads) k_probe_cut(ProbeCutArgs a) {
  __shared__ float lv[kBMaxList];
  __shared__ uint32_t lb[kBMaxList];
  __shared__ __align__(16) uint32_t key[kBMaxList];
  __shared__ uint32_t probe[kBMaxProbes];
  __shared__ float hv[kBMaxList];
  __shared__ int hi[2 * kBMaxList];
  __shared__ long long tmp[32];
  const int tid = threadIdx.x;
  const int q = blockIdx.x;
  const int k = a.q_k ? a.q_k[q] : a.k_uniform;
  const int Qp = a.q_qprobes ? a.q_qprobes[q] : a.qprobes_uniform;
  if (k < 1 || k > a.k_max || Qp < 1 || Qp > a.qprobes_max) {  // the fused kernel rejects the query
    if (tid == 0) a.pc_n[q] = 0;
    return;
  }
  const int L = a.L;
  const int m = (2 * Qp + L - 1) / L;  // ceil(2.0 * qProbes / L), FalconnPP.cpp:336
  const int M = L * m;
  const float* slv = a.ext_lv + (size_t)q * a.ext_stride;
  const uint32_t* slb = a.ext_lb + (size_t)q * a.ext_stride;
  const int M4 = (M + 3) >> 2;
  for (int i = tid; i < 4 * M4; i += kPcThreads) {
    const float v = i < M ? slv[i] : 0.0f;
    if (i < M) {
      lv[i] = v;
      lb[i] = slb[i];
    }
    key[i] = i < M ? ord_key(v) : 0u;  // scores are >= 0: their keys exceed the padding's 0
  }
  __syncthreads();
  long long run = 0;
  bool tie = false;
  for (int base = 0; base < M; base += kPcThreads) {
    const int i = base + tid;
    bool take = false;
    if (i < M) {
      const uint32_t ki = key[i];
      int gt = 0, eq = 0;
      for (int j = 0; j < M4; ++j) {
        const uint4 k4 = reinterpret_cast<const uint4*>(key)[j];
        gt += (k4.x > ki) + (k4.y > ki) + (k4.z > ki) + (k4.w > ki);
        eq += (k4.x == ki) + (k4.y == ki) + (k4.z == ki) + (k4.w == ki);
      }
      take = gt < Qp;
      tie |= take && gt + eq > Qp;
    }
    long long tot;
    const long long pos = block_exclusive_scan(take ? 1 : 0, tmp, &tot) + run;
    if (take && pos < Qp) probe[pos] = lb[i];
    run += tot;
  }
  if (__syncthreads_or(tie) && tid == 0) {
    // a tie at the cut: the reference's max-heap of each table's next list
    // entry, popped qProbes times
    int* track = hi + L;
    int n = 0;
    for (int l = 0; l < L; ++l) {
      heap_push<false, int>(hv, hi, n, lv[l * m], l * m);
      track[l] = 0;
    }
    for (int pc = 0; pc < Qp; ++pc) {
      const int pos = hi[0];
      heap_pop<false, int>(hv, hi, n);
      probe[pc] = lb[pos];
      const int tb = pos / m;
      track[tb]++;
      if (track[tb] < m) heap_push<false, int>(hv, hi, n, lv[tb * m + track[tb]], tb * m + track[tb]);
    }
  }
  __syncthreads();
  const size_t ob = (size_t)q * a.stride;
  run = 0;
  for (int base = 0; base < Qp; base += kPcThreads) {
    const int p = base + tid;
    uint32_t g = 0, o = 0, sz = 0;
    if (p < Qp) {
      g = probe[p];
      o = a.bucket_off[g];
      sz = a.bucket_off[g + 1] - o;
    }
    long long tot;
    const long long ex = block_exclusive_scan((long long)sz, tmp, &tot) + run;
    if (p < Qp) {
      a.pc_g[ob + p] = g;
      a.pc_o[ob + p] = o;
      a.pc_pe[ob + p] = (uint32_t)(ex + sz);
    }
    run += tot;
  }
  if (tid == 0) a.pc_n[q] = Qp;
}

cudaError_t probe_cut_lists(const ProbeCutArgs& a, int nq, cudaStream_t s) {
  if (nq <= 0) return cudaSuccess;
  k_probe_cut<<<nq, kPcThreads, 0, s>>>(a);
  return cudaGetLastError();
}

template <int MODE, int VI, int VI32>
static KernelSel ext_pair(bool big) {
  return big ? kernel_ptr<256, MODE, VI, VI32, kHashExt, true>() : kernel_ptr<256, MODE, VI, VI32, kHashExt, false>();
}

KernelSel pick_kernel_ext(int mode, int d, bool big) {
  const int v32 = vi_of(d, 4);
  if (mode == kRowsF32) {
    if (v32 == 1) return ext_pair<kRowsF32, 1, 1>(big);
    if (v32 == 2) return ext_pair<kRowsF32, 2, 2>(big);
    return ext_pair<kRowsF32, 4, 4>(big);
  }
  if (mode == kRowsBF16) {
    if (v32 == 1) return ext_pair<kRowsBF16, 1, 1>(big);
    if (v32 == 2) return ext_pair<kRowsBF16, 1, 2>(big);
    return ext_pair<kRowsBF16, 1, 4>(big);
  }
  if (v32 == 1) return ext_pair<kRowsFP8, 1, 1>(big);
  if (v32 == 2) return ext_pair<kRowsFP8, 1, 2>(big);
  return ext_pair<kRowsFP8, 1, 4>(big);
}

}  // namespace fpp
