// fpp_batch.h — the batched query form (one persistent fused kernel per batch).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fpp_index.h"

namespace fpp {

struct BatchRequest {
  const float* Q = nullptr;  // device, nq x d
  int nq = 0;
  const int* q_k = nullptr;        // device per-query k (nullable -> k_uniform)
  const int* q_qprobes = nullptr;  // device per-query qProbes (nullable -> qprobes_uniform)
  int k_uniform = 0, qprobes_uniform = 0;
  int k_max = 0, qprobes_max = 0;  // bounds over the batch (scratch sizing)
  int mode = 0;                    // RowMode: 0 fp32 (exact), 1 bf16, 2 fp8
  int shortlist_mult = 4;          // FP32 re-score of shortlist_mult * k candidates
  int32_t* out = nullptr;          // device, nq x out_stride
  int out_stride = 0;
  float* out_v = nullptr;          // optional scores
  bool use_graph = false;
  bool check_status = true;        // synchronise and report overflow
  int blocks_per_sm = 0;           // 0 = as many as fit
  bool reorder = true;             // process the queries grouped by a locality key
  uint32_t* dump_probes = nullptr;  // parity dumps (device, nullable; no graph): [nq][qprobes_max] probes
  uint32_t* dump_counts = nullptr;  // [nq][2] candidates, unique candidates
  bool split_hash = true;           // exact hash in its own kernel before the fused one (kHashExt)
  // split hash, fhtDim 256, L <= 128, 2 qProbes <= L: rotate on the tensor
  // cores and hash again in FP32 every table that can reach the probe cut
  // (k_query_hash_verified); the probes and their scores are unchanged
  bool tc_hash = true;
  // host queries (nullable): batch_query copies them into Q (device, nq x d)
  // itself; with the split hash, in chunks on copy_stream, each chunk's hash
  // launch waiting only for its own chunk, so the copy overlaps the hashing
  const float* Q_host = nullptr;
  cudaStream_t copy_stream = nullptr;
  bool stage_timing = false;        // CUDA events around the hash and the fused kernel (synchronises)
  bool tc_rotation = false;        // opt-in, BF16/FP8, fhtDim 256: rotate on the tensor cores (FP16 operands,
                                   // not the reference's FP32 hash: probes can differ)
};

struct BatchResult {
  int launches = 0;
  int grid = 0;
  bool graph_replayed = false;
  bool overflow = false;
  bool bad_params = false;
  // with stage_timing: the hash kernel (split form), the order and probe-cut
  // kernels, and the fused kernel
  float ms_hash = 0, ms_prep = 0, ms_fused = 0;
  long long tc_exact = 0;           // with stage_timing: tables the verified hash re-hashed in FP32
};

struct BatchKey {
  const float* Q;
  int nq;
  const int* q_k;
  const int* q_qprobes;
  int k_uniform, qprobes_uniform, k_max, qprobes_max, shortlist_mult;
  int32_t* out;
  int out_stride;
  float* out_v;
  int mode, grid;
  const void* kern;
  uint32_t* bitset;
  const uint32_t* order;
  const uint32_t* tflips;
  cudaStream_t stream;
  bool operator==(const BatchKey& o) const {
    return Q == o.Q && nq == o.nq && q_k == o.q_k && q_qprobes == o.q_qprobes && k_uniform == o.k_uniform &&
           qprobes_uniform == o.qprobes_uniform && k_max == o.k_max && qprobes_max == o.qprobes_max && shortlist_mult == o.shortlist_mult && out == o.out &&
           out_stride == o.out_stride && out_v == o.out_v && mode == o.mode && grid == o.grid && kern == o.kern &&
           bitset == o.bitset && order == o.order && tflips == o.tflips && stream == o.stream;
  }
};

// Per-block scratch of the batched kernel (kept between calls) and the cached graph.
struct BatchWorkspace {
  uint32_t* bitset = nullptr;
  long long nwords = 0;
  uint32_t* uniq = nullptr;
  uint32_t* score = nullptr;
  long long cap = 0;
  float* gdump = nullptr;
  float* gheap_v = nullptr;
  int* gheap_i = nullptr;
  int mmax = 0;
  int fht = 0;
  int grid = 0;
  unsigned* counters = nullptr;
  // query order: key per query, histogram of the keys, the permutation
  uint32_t* okey = nullptr;
  uint32_t* ohist = nullptr;
  uint32_t* order = nullptr;
  long long order_cap = 0;
  // big-list form scratch (see BatchArgs)
  float* glv = nullptr;
  uint32_t* glb = nullptr;
  long long list_cap = 0;
  uint32_t* gprobe = nullptr;
  uint32_t* gpo = nullptr;
  uint32_t* gpe = nullptr;
  long long probe_cap = 0;
  float* ggv = nullptr;
  int* ggc = nullptr;
  float* grhv = nullptr;
  int* grhi = nullptr;
  // split hash: per-query lists and the hash kernel's pair-heap scratch
  float* ext_lv = nullptr;
  uint32_t* ext_lb = nullptr;
  long long ext_cap = 0;
  float* hheap_v = nullptr;
  int* hheap_i = nullptr;
  long long hheap_cap = 0;
  // split hash with small lists: k_probe_cut's output per processing slot
  uint32_t* pc_g = nullptr;
  uint32_t* pc_o = nullptr;
  uint32_t* pc_pe = nullptr;
  int* pc_n = nullptr;
  long long pc_cap = 0, pc_ncap = 0;
  cudaEvent_t tev[4] = {nullptr, nullptr, nullptr, nullptr};  // stage timing: start, fused start, end, hash end
  cudaEvent_t cev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // chunked query copy: chunks, start
  cudaGraphExec_t graph_exec = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphNode_t graph_knode = nullptr;
  BatchKey key{};
  void release();
};

// Scratch of the brute-force low-precision block kernel (fpp_bf_lowp.cu):
// query rows, per-query scales, the per-(query, split) shortlist heaps.
struct BfWorkspace {
  unsigned char* qrows = nullptr;
  float* qscale = nullptr;
  unsigned long long* heap = nullptr;
  int* heap_n = nullptr;
  unsigned* status = nullptr;
  size_t cap_q = 0, cap_qs = 0, cap_hv = 0, cap_n = 0;
  void release();
};

int ensure_lowp_rows(const Params& P, DeviceIndex& di, int mode, cudaStream_t s, Error& err);

int batch_query(const Params& P, DeviceIndex& di, BatchWorkspace& bw, const BatchRequest& rq, cudaStream_t s,
                BatchResult& res, Error& err);

}  // namespace fpp
