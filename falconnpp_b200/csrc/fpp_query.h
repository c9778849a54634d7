// fpp_query.h — query pipeline entry point and its reusable device workspace.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "fpp_index.h"

namespace fpp {

// Device buffers kept between calls so repeated queries do not reallocate.
struct QueryWorkspace {
  float* Qd = nullptr;
  size_t cap_Qd = 0;
  float* list_v = nullptr;
  size_t cap_list = 0;
  uint32_t* list_b = nullptr;
  size_t cap_list_b = 0;
  uint32_t* probes = nullptr;
  size_t cap_probes = 0;
  float* probe_v = nullptr;
  size_t cap_probe_v = 0;
  long long* cand = nullptr;
  size_t cap_cand = 0;
  int* empty = nullptr;
  size_t cap_empty = 0;
  long long* n_unique = nullptr;
  size_t cap_nu = 0;
  float* heap_v = nullptr;
  size_t cap_heap_v = 0;
  int* heap_i = nullptr;
  size_t cap_heap_i = 0;
  uint32_t* bitset = nullptr;  // per-block dedupe bitsets, all zero between queries
  int bitset_grid = 0;
  long long bitset_words = 0;
  uint32_t* uniq = nullptr;
  size_t cap_uniq = 0;
  uint32_t* score = nullptr;
  size_t cap_score = 0;
  int32_t* out = nullptr;
  size_t cap_out = 0;
  float* out_v = nullptr;
  size_t cap_out_v = 0;
  int* counters = nullptr;
  size_t cap_counters = 0;
  bool stage_timing = false;
  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  void release();
};

struct QueryStats {
  long long total_cand = 0;    // candidates incl. duplicates
  long long total_unique = 0;  // unique candidates
  long long total_empty = 0;   // probed empty buckets
  long long total_probes = 0;
  int n_select_ties = 0;       // queries whose probe cut needed the exact replay
  int n_topk_ties = 0;         // queries whose top-k needed the exact replay
  long long launches = 0;      // kernels launched by the call
  // CUDA-event durations on the launching stream (only with stage timing on)
  double ms_hash = 0, ms_select = 0, ms_rerank = 0;
  long long tc_exact = 0;  // batched form with stage timing: tables re-hashed in FP32 by the verified hash
};

// Optional host-side dumps for parity checks (any pointer may be null).
struct QueryDumps {
  uint32_t* probes = nullptr;      // [nq][qProbes]
  float* probe_v = nullptr;        // [nq][qProbes]
  float* topk_v = nullptr;         // [nq][k]
  long long* cand_count = nullptr; // [nq]
  long long* unique_count = nullptr;
  bool want_cands = false;         // unique candidate ids per query (unordered)
  std::vector<int32_t> cands;      // out: [nq][cand_stride], valid up to unique_count
  long long cand_stride = 0;
};

// The per-table probe lists of every query (rotate + hash + pair top-m,
// src/FalconnPP.cpp:358-531) with the plain path's kernel, for the batched
// form: q_qprobes (device, nullable: every query uses qp_max) gives each
// query its own m; query q's lists start at list_v / list_b + q * stride.
// heap_v / heap_i: max_groups * ceil(2 qp_max / L) scratch entries.
cudaError_t hash_lists(const Params& P, const DeviceIndex& di, const float* Q, int nq, const int* q_qprobes, int qp_max,
                       float* list_v, uint32_t* list_b, long long stride, float* heap_v, int* heap_i,
                       long long max_groups, cudaStream_t s);

// The same lists for fhtDim 256 when every query keeps one probe per table
// (2 qp_max <= L, L <= 128): the rotations on the tensor cores, and an exact
// FP32 re-hash of every table whose score can reach the probe cut (ties at
// the cut: of every table), so the probe cut selects the same probes with the
// same scores.  n_exact (device, nullable) += the tables re-hashed.
cudaError_t hash_lists_verified(const Params& P, const DeviceIndex& di, const float* Q, int nq, const int* q_qprobes,
                                int qp_max, float* list_v, uint32_t* list_b, long long stride, unsigned* n_exact,
                                cudaStream_t s);

// Queries k_query_hash_verified takes in one full wave of its blocks on the
// current device (SMs x resident blocks x queries per block); 0 if unknown.
long long hash_verified_wave_queries();

int query_index(const Params& P, const DeviceIndex& di, const float* Q, bool q_on_device, int nq, int k,
                int32_t* out, bool out_on_device, QueryWorkspace& ws, QueryStats& st, cudaStream_t s,
                Error& err, QueryDumps* dumps);

}  // namespace fpp
