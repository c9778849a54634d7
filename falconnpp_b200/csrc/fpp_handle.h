// fpp_handle.h — the object behind the opaque fpp_index handle of the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <mutex>
#include <string>

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
  bool params_set = false;
  bool built = false;
  int device = 0;
  cudaStream_t stream = nullptr;
  std::mutex mu;
};

namespace fpp {
int set_last_error(int code, const std::string& msg);  // returns code
int clear_last_error();                                  // returns 0
}  // namespace fpp
