// fpp_handle.h — the object behind the opaque fpp_index handle of the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "fpp_batch.h"
#include "fpp_index.h"
#include "fpp_query.h"

struct fpp_index {
  fpp::Params P;
  fpp::DeviceIndex di;
  fpp::QueryWorkspace ws;
  fpp::HostBits bits;
  fpp::BuildOptions opt;
  fpp::BuildStats bst;
  fpp::QueryStats qst;
  fpp::BatchWorkspace bw;
  fpp::BfWorkspace bfw;
  int form = 0;             // 0 plain three-kernel path, 1 batched fused kernel
  int precision = 0;        // batched form: 0 FP32 (exact), 1 BF16, 2 FP8-E4M3
  int shortlist_mult = 4;   // batched low precision: FP32 re-score of shortlist_mult * k
  bool use_graph = false;   // batched form: capture/replay the launch as a CUDA graph
  int blocks_per_sm = 0;    // batched form: 0 = occupancy limit
  bool reorder = true;      // batched form: process queries grouped by a locality key
  bool tc_hash = true;      // split hash: tensor-core rotation verified by an exact FP32 re-hash near the cut
  bool split_hash = true;   // batched form: exact hash in its own kernel before the fused one
  bool tc_rotation = false;  // opt-in: batched BF16/FP8 tensor-core rotation (FP16 operands; not bit-exact)
  bool params_set = false;
  bool built = false;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t cstream = nullptr;  // host-buffer batched queries: the chunked query copies
  std::mutex mu;
};

namespace fpp {
int set_last_error(int code, const std::string& msg);  // returns code
int clear_last_error();                                  // returns 0
}  // namespace fpp
