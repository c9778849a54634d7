// fpp_index.h — host-side state of one Falconn++ index living in HBM, and the
// internal entry points of the build and query pipelines.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

namespace fpp {

// Status codes returned through the C ABI.
enum Status : int {
  kOk = 0,
  kErrInvalidArgument = -1,
  kErrNotBuilt = -2,
  kErrCuda = -3,
  kErrOutOfMemory = -4,
  kErrUnsupported = -5,
  kErrNonFinite = -6,
  kErrDevice = -7,
};

struct Error {
  int code;
  std::string msg;
};

// Every device allocation of the library goes through dev_malloc.  For
// fault-injection tests on the host, arm_alloc_failure(n) (n >= 1) makes the
// n-th allocation from then on fail with cudaErrorMemoryAllocation, once,
// without calling cudaMalloc; n = 0 disarms it.  Process-wide.
cudaError_t dev_malloc_bytes(void** p, size_t bytes);
template <typename T>
inline cudaError_t dev_malloc(T** p, size_t bytes) {
  return dev_malloc_bytes(reinterpret_cast<void**>(p), bytes);
}
void arm_alloc_failure(long long nth);

// Parameters mirror FalconnPP's members (src/FalconnPP.h:14-39).
struct Params {
  int n_points = 0;
  int n_features = 0;
  int n_tables = 10;
  int n_proj = 512;
  int n_rotate = 3;
  int n_threads = -1;
  int bucket_minSize = 50;
  float bucket_scale = 1.0f;
  int iProbes = 1;
  int qProbes = 1;
  long long seed = -1;
  int fhtDim = 0;
};

// Reranking precision of the query path.
enum RerankMode : int { kRerankFP32 = 0, kRerankBF16 = 1, kRerankFP8 = 2 };

struct DeviceIndex {
  // centred data, point-major, row stride ld floats (ld = d rounded up to 4)
  float* Xc = nullptr;
  int ld = 0;
  float* center = nullptr;           // d floats
  uint32_t* flips = nullptr;         // [2][L][3][words]: 1 = negate (bitHD == 0)
  uint32_t* tflips = nullptr;        // fhtDim 256 only: the same words per rotation view
                                     // (round 2 holds the transposed 16 x 16 bit matrix)
  uint32_t* bucket_off = nullptr;    // L*4D^2 + 1 CSR offsets into ids
  int32_t* ids = nullptr;            // stored ids, bucket after bucket
  uint64_t n_ids = 0;
  uint32_t max_kept = 0;
  // low-precision copies for the precision form
  void* Xlp = nullptr;               // bf16 [n][ld] or fp8 [n][ld8]
  float* Xlp_scale = nullptr;        // per-row FP32 scale (fp8)
  int lp_mode = kRerankFP32;
  int ld_lp = 0;
};

struct BuildStats {
  double ms_center = 0, ms_hash = 0, ms_sort = 0, ms_csr = 0, ms_total = 0;
  long long n_repaired = 0;
  long long n_limited = 0;
  double points_per_table = 0;  // sum kept / n / L  (FalconnPP.cpp:268, :296)
};

struct HostBits {
  std::vector<uint8_t> b1, b2;  // bitHD1/bitHD2 as in src/FalconnPP.h:61-68
};

// Options that only tests and tools change.
struct BuildOptions {
  bool exact_bucket_order = true;  // replay ties inside kept prefixes too
  int tables_per_chunk = 0;        // 0 = automatic
};

int build_index(const Params& P, const float* X, bool x_on_device, const HostBits& bits,
                const BuildOptions& opt, DeviceIndex& di, BuildStats& st, cudaStream_t s, Error& err,
                int32_t* dump_codes, float* dump_scores);

void free_index(DeviceIndex& di);

// The sign flip words (and, for fhtDim 256, their per-view copy for the
// tensor-core rotation) from the sign bits, into di.flips / di.tflips;
// synchronises s before returning.
int upload_flips(const Params& P, const HostBits& bits, DeviceIndex& di, cudaStream_t s, Error& err);

int derived_fht_dim(int n_features, int n_proj);

}  // namespace fpp
