// fpp_capi.cu — the extern "C" boundary (include/falconnpp_b200.h) over the
// device index: parameter handling as in FalconnPP::Index2Layers
// (src/FalconnPP.h:85-123), the random signs of bitHD3Generator2
// (src/FalconnPP.h:52-75, same libstdc++ engine and distribution), status
// codes instead of undefined behaviour, and the verbose side effects of
// query2Layers_1D (src/FalconnPP.cpp:682-703).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <atomic>
#include <chrono>
#include <fstream>
#include <iostream>
#include <mutex>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/falconnpp_b200.h"
#include "fpp_index.h"
#include "fpp_query.h"

#include "fpp_handle.h"

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int ok() {
  g_last_error.clear();
  return FPP_OK;
}

bool is_pow2(int x) { return x > 0 && (x & (x - 1)) == 0; }

// src/FalconnPP.h:52-68: one default_random_engine, two draws per position.
void generate_bits(const fpp::Params& P, fpp::HostBits& b) {
  const int nbits = P.fhtDim * P.n_tables * P.n_rotate;
  unsigned seed = std::chrono::system_clock::now().time_since_epoch().count();
  if (P.seed > -1) seed = (unsigned)P.seed;
  std::default_random_engine generator(seed);
  std::uniform_int_distribution<uint32_t> unifDist(0, 1);
  b.b1.assign(nbits, 0);
  b.b2.assign(nbits, 0);
  for (int d = 0; d < nbits; ++d) {
    b.b1[d] = unifDist(generator) & 1;
    b.b2[d] = unifDist(generator) & 1;
  }
}

int use_device(fpp_index* h) {
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return fail(FPP_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  return FPP_OK;
}

int check_query_params(const fpp_index* h, int n_queries, int k) {
  if (!h->built) return fail(FPP_ERR_NOT_BUILT, "query: the index is not built");
  if (n_queries < 0) return fail(FPP_ERR_INVALID_ARGUMENT, "query: n_queries must be >= 0");
  if (k < 1 || k > 1024) return fail(FPP_ERR_INVALID_ARGUMENT, "query: n_neighbors must be in [1, 1024]");
  const fpp::Params& P = h->P;
  if (P.qProbes < 1) return fail(FPP_ERR_INVALID_ARGUMENT, "query: qProbes must be >= 1");
  const int m = (int)ceil(2.0 * P.qProbes / P.n_tables);
  const int m1 = (int)ceil(sqrt(1.0 * m));
  if (m1 > P.n_proj || m1 > 64)
    return fail(FPP_ERR_INVALID_ARGUMENT,
                "query: qProbes too large: ceil(sqrt(ceil(2*qProbes/n_tables))) must be <= min(n_proj, 64)");
  if ((long long)P.n_tables * m > (1LL << 24))
    return fail(FPP_ERR_INVALID_ARGUMENT, "query: n_tables * probes per table too large");
  return FPP_OK;
}

std::string int2str(int x) {
  std::stringstream ss;
  ss << x;
  return ss.str();
}

int do_build(fpp_index* h, const float* X, bool on_device, cudaStream_t s, int32_t* codes_host, float* scores_host) {
  if (!h->params_set) return fail(FPP_ERR_INVALID_ARGUMENT, "build: call setIndexParam first");
  if (!X) return fail(FPP_ERR_INVALID_ARGUMENT, "build: dataset is NULL");
  if (use_device(h)) return FPP_ERR_CUDA;
  fpp::Params& P = h->P;
  generate_bits(P, h->bits);
  int32_t* dcodes = nullptr;
  float* dscores = nullptr;
  const size_t ncodes = (size_t)P.n_tables * P.n_points * P.iProbes;
  if (codes_host) {
    if (fpp::dev_malloc(&dcodes, sizeof(int32_t) * ncodes) != cudaSuccess ||
        fpp::dev_malloc(&dscores, sizeof(float) * ncodes) != cudaSuccess) {
      cudaFree(dcodes);
      return fail(FPP_ERR_OUT_OF_MEMORY, "build: cannot allocate the hash-code dump");
    }
  }
  h->ws.release();
  h->bw.release();
    h->bfw.release();
  h->built = false;
  fpp::Error err{0, ""};
  h->bst = fpp::BuildStats();
  const int rc = fpp::build_index(P, X, on_device, h->bits, h->opt, h->di, h->bst, s, err, dcodes, dscores);
  if (rc == FPP_OK && codes_host) {
    cudaMemcpy(codes_host, dcodes, sizeof(int32_t) * ncodes, cudaMemcpyDeviceToHost);
    cudaMemcpy(scores_host, dscores, sizeof(float) * ncodes, cudaMemcpyDeviceToHost);
  }
  cudaFree(dcodes);
  cudaFree(dscores);
  if (rc != FPP_OK) return fail(rc, err.msg);
  h->built = true;
  return ok();
}

void print_build(const fpp_index* h) {
  // src/FalconnPP.cpp:23-30 and :281-301
  const fpp::Params& P = h->P;
  std::cout << "n_points: " << P.n_points << std::endl;
  std::cout << "n_features: " << P.n_features << std::endl;
  std::cout << "n_tables: " << P.n_tables << std::endl;
  std::cout << "n_proj: " << P.n_proj << std::endl;
  std::cout << "fhtDim: " << P.fhtDim << std::endl;
  std::cout << "# iProbes: " << P.iProbes << std::endl;
  std::cout << "bucket_minSize: " << P.bucket_minSize << std::endl;
  std::cout << "bucket_scale: " << P.bucket_scale << std::endl;
  std::cout << "Finish building index... " << std::endl;
  const double nb = 4.0 * P.n_proj * P.n_proj * P.n_tables;
  const double size_1d = 1.0 * sizeof(int32_t) * h->di.n_ids / (1 << 30);
  const double size_pos = 1.0 * sizeof(uint32_t) * (nb + 1) / (1 << 30);
  std::cout << "Size of vecTables_1D in GB: " << size_1d << std::endl;
  std::cout << "Size of vecPair_BucketPos in GB: " << size_pos << std::endl;
  std::cout << "Size of Falconn++ (2 layers) index in GB: " << size_1d + size_pos << std::endl;
  std::cout << "n_points per table / n: " << h->bst.points_per_table << std::endl;
  std::cout << "Percentage of scaled buckets in a table: " << 1.0 * h->bst.n_limited / nb << std::endl;
  std::cout << "Construct Falconn++ (2 layers) Wall Time (in seconds): " << (float)(int)(h->bst.ms_total / 1000.0)
            << " seconds" << std::endl;
}

// The query statistics of a batched call: kernels launched and, with
// "stage_timing", the CUDA-event milliseconds of the hash kernel (split form),
// the order and probe-cut kernels and the fused gather / rerank / top-k
// kernel, and the tables the verified tensor-core hash re-hashed in FP32.
void set_batch_stats(fpp_index* h, const fpp::BatchResult& res) {
  h->qst = fpp::QueryStats();
  h->qst.launches = res.launches;
  h->qst.ms_hash = res.ms_hash;
  h->qst.ms_select = res.ms_prep;
  h->qst.ms_rerank = res.ms_fused;
  h->qst.tc_exact = res.tc_exact;
}

// Runs the batched form for device queries/outputs (uniform k, the handle's
// qProbes).  With check_status false the call does not wait for the kernel;
// the caller reads the status words (h->bw.counters + 1) after its own copies
// and reports an overflow with batched_overflow_error().
int run_batched(fpp_index* h, const float* dQ, int nq, int k, int32_t* dout, cudaStream_t s,
                bool check_status = true, const float* Q_host = nullptr, cudaStream_t copy_stream = nullptr) {
  fpp::BatchRequest rq;
  rq.Q = dQ;
  rq.Q_host = Q_host;
  rq.copy_stream = copy_stream;
  rq.nq = nq;
  rq.k_uniform = k;
  rq.qprobes_uniform = h->P.qProbes;
  rq.k_max = k;
  rq.qprobes_max = h->P.qProbes;
  rq.mode = h->precision;
  rq.shortlist_mult = h->shortlist_mult;
  rq.out = dout;
  rq.out_stride = k;
  rq.use_graph = h->use_graph;
  rq.blocks_per_sm = h->blocks_per_sm;
  rq.reorder = h->reorder;
  rq.tc_rotation = h->tc_rotation;
  rq.split_hash = h->split_hash;
  rq.tc_hash = h->tc_hash;
  rq.stage_timing = h->ws.stage_timing;
  rq.check_status = check_status;
  fpp::BatchResult res;
  fpp::Error err{0, ""};
  const int rc = fpp::batch_query(h->P, h->di, h->bw, rq, s, res, err);
  if (rc) return fail(rc, err.msg);
  if (res.overflow) return fail(FPP_ERR_UNSUPPORTED, "batched query: candidate capacity exceeded");
  set_batch_stats(h, res);
  h->qst.total_probes = (long long)nq * h->P.qProbes;
  return FPP_OK;
}

}  // namespace

namespace fpp {
// Lets the other translation units of the library report an error through
// fpp_last_error().
int set_last_error(int code, const std::string& msg) { return fail(code, msg); }
int clear_last_error() { return ok(); }

static std::atomic<long long> g_alloc_countdown{0};

cudaError_t dev_malloc_bytes(void** p, size_t bytes) {
  long long c = g_alloc_countdown.load();
  while (c > 0 && !g_alloc_countdown.compare_exchange_weak(c, c - 1)) {
  }
  if (c == 1) {  // this is the armed allocation: fail it on the host
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(p, bytes);
}

void arm_alloc_failure(long long nth) { g_alloc_countdown.store(nth > 0 ? nth : 0); }
}  // namespace fpp

extern "C" {

const char* fpp_last_error(void) { return g_last_error.c_str(); }

int fpp_create(int n_points, int n_features, fpp_index** out) {
  if (!out) return fail(FPP_ERR_INVALID_ARGUMENT, "create: out is NULL");
  *out = nullptr;
  if (n_points < 1) return fail(FPP_ERR_INVALID_ARGUMENT, "create: n_points must be >= 1");
  if (n_features < 1) return fail(FPP_ERR_INVALID_ARGUMENT, "create: n_features must be >= 1");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(FPP_ERR_DEVICE, std::string("create: no CUDA device: ") + cudaGetErrorString(e));
  fpp_index* h = new fpp_index();
  h->P.n_points = n_points;
  h->P.n_features = n_features;
  h->device = dev;
  e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete h;
    return fail(FPP_ERR_CUDA, std::string("create: cudaStreamCreate: ") + cudaGetErrorString(e));
  }
  *out = h;
  return ok();
}

void fpp_destroy(fpp_index* h) {
  if (!h) return;
  {
    std::lock_guard<std::mutex> g(h->mu);
    cudaSetDevice(h->device);
    h->ws.release();
    h->bw.release();
    h->bfw.release();
    fpp::free_index(h->di);
    if (h->stream) cudaStreamDestroy(h->stream);
    if (h->cstream) cudaStreamDestroy(h->cstream);
  }
  delete h;
}

int fpp_set_index_param(fpp_index* h, int n_tables, int n_proj, int bucket_minSize, float bucket_scale,
                        int iProbes, int n_threads, int random_seed) {
  if (!h) return fail(FPP_ERR_INVALID_ARGUMENT, "setIndexParam: NULL handle");
  std::lock_guard<std::mutex> g(h->mu);
  if (n_tables < 1) return fail(FPP_ERR_INVALID_ARGUMENT, "setIndexParam: n_tables must be >= 1");
  if (!is_pow2(n_proj)) return fail(FPP_ERR_INVALID_ARGUMENT, "setIndexParam: n_proj must be a power of two");
  const int fht = fpp::derived_fht_dim(h->P.n_features, n_proj);
  if (fht > 1024 || n_proj > 1024)
    return fail(FPP_ERR_UNSUPPORTED, "setIndexParam: fhtDim = 2^ceil(log2(max(d, n_proj))) must be <= 1024");
  if (fht < 2) return fail(FPP_ERR_UNSUPPORTED, "setIndexParam: fhtDim must be >= 2");
  if (iProbes < 1 || iProbes > 32 || iProbes > n_proj)
    return fail(FPP_ERR_INVALID_ARGUMENT, "setIndexParam: iProbes must be in [1, min(32, n_proj)]");
  if (!(bucket_scale >= 0.0f) || !isfinite(bucket_scale))
    return fail(FPP_ERR_INVALID_ARGUMENT, "setIndexParam: bucket_scale must be finite and >= 0");
  if ((long long)n_tables * 4LL * n_proj * n_proj >= (1LL << 31))
    return fail(FPP_ERR_UNSUPPORTED, "setIndexParam: n_tables * 4 * n_proj^2 must be < 2^31 (int bucket ids)");
  fpp::Params& P = h->P;
  P.n_tables = n_tables;
  P.n_proj = n_proj;
  P.bucket_minSize = bucket_minSize;
  P.bucket_scale = bucket_scale;
  P.iProbes = iProbes;
  P.n_threads = n_threads;
  P.seed = random_seed;
  P.fhtDim = fht;
  h->params_set = true;
  return ok();
}

int fpp_set_qprobes(fpp_index* h, int qProbes) {
  if (!h) return fail(FPP_ERR_INVALID_ARGUMENT, "set_qProbes: NULL handle");
  if (qProbes < 1) return fail(FPP_ERR_INVALID_ARGUMENT, "set_qProbes: qProbes must be >= 1");
  std::lock_guard<std::mutex> g(h->mu);
  h->P.qProbes = qProbes;
  return ok();
}

int fpp_set_threads(fpp_index* h, int n_threads) {
  if (!h) return fail(FPP_ERR_INVALID_ARGUMENT, "set_threads: NULL handle");
  std::lock_guard<std::mutex> g(h->mu);
  h->P.n_threads = n_threads;
  return ok();
}

int fpp_clear(fpp_index* h) {
  if (!h) return fail(FPP_ERR_INVALID_ARGUMENT, "clear: NULL handle");
  std::lock_guard<std::mutex> g(h->mu);
  cudaSetDevice(h->device);
  h->ws.release();
  h->bw.release();
    h->bfw.release();
  fpp::free_index(h->di);
  h->bits = fpp::HostBits();
  h->built = false;
  return ok();
}

int fpp_set_option(fpp_index* h, const char* key, long long value) {
  if (!h || !key) return fail(FPP_ERR_INVALID_ARGUMENT, "set_option: NULL argument");
  std::lock_guard<std::mutex> g(h->mu);
  if (!strcmp(key, "exact_bucket_order")) {
    h->opt.exact_bucket_order = value != 0;
  } else if (!strcmp(key, "use_graph")) {
    h->use_graph = value != 0;
  } else if (!strcmp(key, "reorder_queries")) {
    h->reorder = value != 0;
  } else if (!strcmp(key, "tc_rotation")) {
    h->tc_rotation = value != 0;
  } else if (!strcmp(key, "split_hash")) {
    h->split_hash = value != 0;
  } else if (!strcmp(key, "tc_hash")) {
    h->tc_hash = value != 0;
  } else if (!strcmp(key, "blocks_per_sm")) {
    if (value < 0) return fail(FPP_ERR_INVALID_ARGUMENT, "set_option: blocks_per_sm must be >= 0");
    h->blocks_per_sm = (int)value;
  } else if (!strcmp(key, "stage_timing")) {
    h->ws.stage_timing = value != 0;
  } else if (!strcmp(key, "inject_alloc_failure")) {
    if (value < 0) return fail(FPP_ERR_INVALID_ARGUMENT, "set_option: inject_alloc_failure must be >= 0");
    fpp::arm_alloc_failure(value);
  } else if (!strcmp(key, "tables_per_chunk")) {
    if (value < 0) return fail(FPP_ERR_INVALID_ARGUMENT, "set_option: tables_per_chunk must be >= 0");
    h->opt.tables_per_chunk = (int)value;
  } else {
    return fail(FPP_ERR_INVALID_ARGUMENT, std::string("set_option: unknown key ") + key);
  }
  return ok();
}

int fpp_build(fpp_index* h, const float* dataset) {
  if (!h) return fail(FPP_ERR_INVALID_ARGUMENT, "build: NULL handle");
  std::lock_guard<std::mutex> g(h->mu);
  const int rc = do_build(h, dataset, false, h->stream, nullptr, nullptr);
  return rc;
}

int fpp_build_device(fpp_index* h, const float* d_dataset, void* stream) {
  if (!h) return fail(FPP_ERR_INVALID_ARGUMENT, "build: NULL handle");
  std::lock_guard<std::mutex> g(h->mu);
  cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
  return do_build(h, d_dataset, true, s, nullptr, nullptr);
}

int fpp_build_dump_hash(fpp_index* h, const float* dataset, int32_t* codes, float* scores) {
  if (!h || !codes || !scores) return fail(FPP_ERR_INVALID_ARGUMENT, "build_dump_hash: NULL argument");
  std::lock_guard<std::mutex> g(h->mu);
  return do_build(h, dataset, false, h->stream, codes, scores);
}

int fpp_query(fpp_index* h, const float* queries, int n_queries, int n_neighbors, int verbose, int32_t* out) {
  if (!h) return fail(FPP_ERR_INVALID_ARGUMENT, "query: NULL handle");
  std::lock_guard<std::mutex> g(h->mu);
  int rc = check_query_params(h, n_queries, n_neighbors);
  if (rc) return rc;
  if (n_queries > 0 && (!queries || !out)) return fail(FPP_ERR_INVALID_ARGUMENT, "query: NULL buffer");
  if (use_device(h)) return FPP_ERR_CUDA;
  const fpp::Params& P = h->P;
  if (verbose) {
    std::cout << "number of queries: " << n_queries << std::endl;
    std::cout << "# qProbes: " << P.qProbes << std::endl;
    std::cout << "number of threads: " << P.n_threads << std::endl;
  }
  const auto t0 = std::chrono::high_resolution_clock::now();
  fpp::Error err{0, ""};
  if (h->form == 1 && n_queries > 0) {
    // batched form: stage the queries and results through the workspace
    size_t capq = h->ws.cap_Qd, capo = h->ws.cap_out;
    cudaError_t e = cudaSuccess;
    if ((size_t)n_queries * P.n_features > capq) {
      cudaFree(h->ws.Qd);
      h->ws.Qd = nullptr;
      h->ws.cap_Qd = 0;
      e = fpp::dev_malloc(&h->ws.Qd, sizeof(float) * n_queries * P.n_features);
      if (e == cudaSuccess) h->ws.cap_Qd = (size_t)n_queries * P.n_features;
    }
    if (e == cudaSuccess && (size_t)n_queries * n_neighbors > capo) {
      cudaFree(h->ws.out);
      h->ws.out = nullptr;
      h->ws.cap_out = 0;
      e = fpp::dev_malloc(&h->ws.out, sizeof(int32_t) * n_queries * n_neighbors);
      if (e == cudaSuccess) h->ws.cap_out = (size_t)n_queries * n_neighbors;
    }
    if (e != cudaSuccess) return fail(FPP_ERR_OUT_OF_MEMORY, std::string("query: ") + cudaGetErrorString(e));
    if (!h->cstream && cudaStreamCreateWithFlags(&h->cstream, cudaStreamNonBlocking) != cudaSuccess)
      h->cstream = nullptr;
    // the queries are copied by the batched form itself (in chunks that
    // overlap the hashing); one synchronisation: results and the kernel's
    // status words come back together
    rc = run_batched(h, h->ws.Qd, n_queries, n_neighbors, h->ws.out, h->stream, false, queries, h->cstream);
    if (rc) return rc;
    unsigned status = 0;
    e = cudaMemcpyAsync(out, h->ws.out, sizeof(int32_t) * n_queries * n_neighbors, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(&status, h->bw.counters + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return fail(FPP_ERR_CUDA, std::string("query: ") + cudaGetErrorString(e));
    if (status & 1u) return fail(FPP_ERR_UNSUPPORTED, "batched query: candidate capacity exceeded");
  } else {
    rc = fpp::query_index(P, h->di, queries, false, n_queries, n_neighbors, out, false, h->ws, h->qst, h->stream,
                          err, nullptr);
    if (rc) return fail(rc, err.msg);
  }
  if (verbose && n_queries > 0) {
    const auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::high_resolution_clock::now() - t0);
    const fpp::QueryStats& s = h->qst;
    std::cout << "Average number of empty buckets per query: " << (float)s.total_empty / n_queries << std::endl;
    std::cout << "Average number of probes per query: " << (float)s.total_probes / n_queries << std::endl;
    std::cout << "Average number of unique candidates per query: " << (float)s.total_unique / n_queries << std::endl;
    std::cout << "Average number of candidates per query: " << (float)s.total_cand / n_queries << std::endl;
    std::cout << "Querying Time: " << (float)ms.count() << " ms" << std::endl;
    const std::string fn = "1D_Top_" + int2str(n_neighbors) + "_D_" + int2str(P.n_proj) + "_L_" +
                           int2str(P.n_tables) + "_iProbe_" + int2str(P.iProbes) + "_bucketMinSize_" +
                           int2str(P.bucket_minSize) + "_bucketScale_" + int2str((int)(P.bucket_scale * 100)) +
                           "_qProbe_" + int2str(P.qProbes) + ".txt";
    std::ofstream f(fn);  // src/Utilities.cpp:13-33: one query per line
    for (int q = 0; q < n_queries; ++q) {
      for (int j = 0; j < n_neighbors; ++j) f << out[(size_t)q * n_neighbors + j] << ' ';
      f << '\n';
    }
  }
  return ok();
}

int fpp_query_device(fpp_index* h, const float* d_queries, int n_queries, int n_neighbors, int32_t* d_out,
                     void* stream) {
  if (!h) return fail(FPP_ERR_INVALID_ARGUMENT, "query: NULL handle");
  std::lock_guard<std::mutex> g(h->mu);
  int rc = check_query_params(h, n_queries, n_neighbors);
  if (rc) return rc;
  if (n_queries > 0 && (!d_queries || !d_out)) return fail(FPP_ERR_INVALID_ARGUMENT, "query: NULL buffer");
  if (use_device(h)) return FPP_ERR_CUDA;
  cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
  fpp::Error err{0, ""};
  if (h->form == 1) {
    rc = run_batched(h, d_queries, n_queries, n_neighbors, d_out, s);
    if (rc) return rc;
    return ok();
  }
  rc = fpp::query_index(h->P, h->di, d_queries, true, n_queries, n_neighbors, d_out, true, h->ws, h->qst, s, err,
                        nullptr);
  if (rc) return fail(rc, err.msg);
  return ok();
}

int fpp_set_query_form(fpp_index* h, int form, int precision, int shortlist_mult) {
  if (!h) return fail(FPP_ERR_INVALID_ARGUMENT, "set_query_form: NULL handle");
  if (form < 0 || form > 1) return fail(FPP_ERR_INVALID_ARGUMENT, "set_query_form: form must be 0 or 1");
  if (precision < 0 || precision > 2) return fail(FPP_ERR_INVALID_ARGUMENT, "set_query_form: precision must be 0..2");
  if (shortlist_mult < 1 || shortlist_mult > 64)
    return fail(FPP_ERR_INVALID_ARGUMENT, "set_query_form: shortlist_mult must be in [1, 64]");
  if (form == 0 && precision != 0)
    return fail(FPP_ERR_INVALID_ARGUMENT, "set_query_form: the plain form is FP32 only");
  std::lock_guard<std::mutex> g(h->mu);
  h->form = form;
  h->precision = precision;
  h->shortlist_mult = shortlist_mult;
  return ok();
}

int fpp_autotune(fpp_index* h, const float* d_queries, int n_queries, int k, double min_agreement, double* report,
                 void* stream) {
  if (!h) return fail(FPP_ERR_INVALID_ARGUMENT, "autotune: NULL handle");
  std::lock_guard<std::mutex> g(h->mu);
  if (!h->built) return fail(FPP_ERR_NOT_BUILT, "autotune: the index is not built");
  if (n_queries < 1 || k < 1 || k > 1024 || !d_queries)
    return fail(FPP_ERR_INVALID_ARGUMENT, "autotune: need queries and 1 <= k <= 1024");
  if (use_device(h)) return FPP_ERR_CUDA;
  cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
  const size_t nout = (size_t)n_queries * k;
  int32_t* d_ref = nullptr;
  int32_t* d_out = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (fpp::dev_malloc(&d_ref, sizeof(int32_t) * nout) != cudaSuccess ||
      fpp::dev_malloc(&d_out, sizeof(int32_t) * nout) != cudaSuccess) {
    cudaFree(d_ref);
    return fail(FPP_ERR_OUT_OF_MEMORY, "autotune: cannot allocate result buffers");
  }
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  std::vector<int32_t> ref(nout), got(nout);
  auto run = [&](int precision, int mult, int bps, bool split, bool reorder, int32_t* out, float* ms) -> int {
    fpp::BatchRequest rq;
    rq.Q = d_queries;
    rq.nq = n_queries;
    rq.k_uniform = k;
    rq.qprobes_uniform = h->P.qProbes;
    rq.k_max = k;
    rq.qprobes_max = h->P.qProbes;
    rq.mode = precision;
    rq.shortlist_mult = mult;
    rq.out = out;
    rq.out_stride = k;
    rq.blocks_per_sm = bps;
    rq.reorder = reorder;
    rq.tc_rotation = h->tc_rotation;
    rq.split_hash = split;
    rq.tc_hash = h->tc_hash;
    rq.check_status = true;
    fpp::BatchResult res;
    fpp::Error err{0, ""};
    int rc = fpp::batch_query(h->P, h->di, h->bw, rq, s, res, err);  // warm-up, checks status
    if (rc) return fail(rc, err.msg);
    if (res.overflow || res.bad_params) return fail(FPP_ERR_UNSUPPORTED, "autotune: batch did not complete");
    float best = 1e30f;
    rq.check_status = false;
    for (int rep = 0; rep < 3; ++rep) {
      cudaEventRecord(e0, s);
      rc = fpp::batch_query(h->P, h->di, h->bw, rq, s, res, err);
      cudaEventRecord(e1, s);
      if (rc) return fail(rc, err.msg);
      cudaEventSynchronize(e1);
      float t = 0;
      cudaEventElapsedTime(&t, e0, e1);
      best = std::min(best, t);
    }
    *ms = best;
    return FPP_OK;
  };
  float ms = 0;
  int rc = run(0, 1, 0, true, h->reorder, d_ref, &ms);
  double best_ms = 1e30, best_agree = 0;
  int best_bps = 0, best_prec = 0, best_mult = 4, tried = 0;
  bool best_split = true, best_reorder = h->reorder;
  if (rc == FPP_OK) {
    cudaMemcpy(ref.data(), d_ref, sizeof(int32_t) * nout, cudaMemcpyDeviceToHost);
    best_ms = ms;
    best_agree = 1.0;
    const int precs[2] = {1, 2};
    const int mults[2] = {2, 4};  // the exact FP32 re-score of a 2-4 x k shortlist
    const int bpss[3] = {1, 2, 3};
    // precision x shortlist x resident blocks per SM (queries in flight per
    // SM) x exact hash in its own kernel or inside the fused one x query
    // grouping; the hash and grouping choices change no result
    for (int pi = 0; pi < 2 && rc == FPP_OK; ++pi)
      for (int mi = 0; mi < 2 && rc == FPP_OK; ++mi)
        for (int bi = 0; bi < 3 && rc == FPP_OK; ++bi)
          for (int sp = 1; sp >= 0 && rc == FPP_OK; --sp)
            for (int ro = 1; ro >= 0 && rc == FPP_OK; --ro) {
          if ((long long)k * mults[mi] > 1024) continue;
          rc = run(precs[pi], mults[mi], bpss[bi], sp != 0, ro != 0, d_out, &ms);
          if (rc) break;
          ++tried;
          cudaMemcpy(got.data(), d_out, sizeof(int32_t) * nout, cudaMemcpyDeviceToHost);
          long long hit = 0;
          for (int q = 0; q < n_queries; ++q) {
            const int32_t* a = &ref[(size_t)q * k];
            const int32_t* b = &got[(size_t)q * k];
            for (int i = 0; i < k; ++i)
              for (int j = 0; j < k; ++j)
                if (a[i] == b[j]) {
                  ++hit;
                  break;
                }
          }
          const double agree = (double)hit / (double)nout;
          if (agree >= min_agreement && ms < best_ms) {
            best_ms = ms;
            best_agree = agree;
            best_bps = bpss[bi];
            best_prec = precs[pi];
            best_mult = mults[mi];
            best_split = sp != 0;
            best_reorder = ro != 0;
          }
        }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d_ref);
  cudaFree(d_out);
  if (rc) return rc;
  h->form = 1;
  h->precision = best_prec;
  h->shortlist_mult = best_mult;
  h->blocks_per_sm = best_bps;
  h->split_hash = best_split;
  h->reorder = best_reorder;
  if (report) {
    report[0] = best_ms;
    report[1] = best_bps;
    report[2] = best_prec;
    report[3] = best_mult;
    report[4] = best_agree;
    report[5] = tried;
    report[6] = best_split ? 1 : 0;
    report[7] = best_reorder ? 1 : 0;
  }
  return ok();
}

int fpp_query_batched(fpp_index* h, const float* d_queries, int n_queries, const int32_t* d_k,
                      const int32_t* d_qprobes, int k_max, int qprobes_max, int32_t* d_out, int out_stride,
                      float* d_out_val, void* stream) {
  if (!h) return fail(FPP_ERR_INVALID_ARGUMENT, "query_batched: NULL handle");
  std::lock_guard<std::mutex> g(h->mu);
  if (!h->built) return fail(FPP_ERR_NOT_BUILT, "query_batched: the index is not built");
  if (n_queries < 0 || k_max < 1 || k_max > 1024 || qprobes_max < 1 || out_stride < k_max)
    return fail(FPP_ERR_INVALID_ARGUMENT, "query_batched: bad sizes (need 1 <= k <= 1024, out_stride >= k_max)");
  if (n_queries == 0) return ok();
  if (!d_queries || !d_out) return fail(FPP_ERR_INVALID_ARGUMENT, "query_batched: NULL buffer");
  if (use_device(h)) return FPP_ERR_CUDA;
  cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
  fpp::BatchRequest rq;
  rq.Q = d_queries;
  rq.nq = n_queries;
  rq.q_k = d_k;
  rq.q_qprobes = d_qprobes;
  rq.k_uniform = k_max;
  rq.qprobes_uniform = qprobes_max;
  rq.k_max = k_max;
  rq.qprobes_max = qprobes_max;
  rq.mode = h->precision;
  rq.shortlist_mult = h->shortlist_mult;
  rq.out = d_out;
  rq.out_stride = out_stride;
  rq.out_v = d_out_val;
  rq.use_graph = h->use_graph;
  rq.blocks_per_sm = h->blocks_per_sm;
  rq.reorder = h->reorder;
  rq.tc_rotation = h->tc_rotation;
  rq.split_hash = h->split_hash;
  rq.tc_hash = h->tc_hash;
  rq.check_status = true;
  fpp::BatchResult res;
  fpp::Error err{0, ""};
  const int rc = fpp::batch_query(h->P, h->di, h->bw, rq, s, res, err);
  if (rc) return fail(rc, err.msg);
  if (res.overflow) return fail(FPP_ERR_UNSUPPORTED, "query_batched: candidate capacity exceeded");
  if (res.bad_params)
    return fail(FPP_ERR_INVALID_ARGUMENT, "query_batched: a per-query k or qProbes is outside [1, k_max/qprobes_max]");
  set_batch_stats(h, res);
  return ok();
}

int fpp_query_batched_dump(fpp_index* h, const float* d_queries, int n_queries, int n_neighbors, int32_t* d_out,
                           float* d_out_val, uint32_t* d_probes, uint32_t* d_counts, void* stream) {
  if (!h) return fail(FPP_ERR_INVALID_ARGUMENT, "query_batched_dump: NULL handle");
  std::lock_guard<std::mutex> g(h->mu);
  int rc = check_query_params(h, n_queries, n_neighbors);
  if (rc) return rc;
  if (n_queries == 0) return ok();
  if (!d_queries || !d_out) return fail(FPP_ERR_INVALID_ARGUMENT, "query_batched_dump: NULL buffer");
  if (use_device(h)) return FPP_ERR_CUDA;
  cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
  fpp::BatchRequest rq;
  rq.Q = d_queries;
  rq.nq = n_queries;
  rq.k_uniform = n_neighbors;
  rq.qprobes_uniform = h->P.qProbes;
  rq.k_max = n_neighbors;
  rq.qprobes_max = h->P.qProbes;
  rq.mode = h->precision;
  rq.shortlist_mult = h->shortlist_mult;
  rq.out = d_out;
  rq.out_stride = n_neighbors;
  rq.out_v = d_out_val;
  rq.blocks_per_sm = h->blocks_per_sm;
  rq.reorder = h->reorder;
  rq.tc_rotation = h->tc_rotation;
  rq.split_hash = h->split_hash;
  rq.tc_hash = h->tc_hash;
  rq.dump_probes = d_probes;
  rq.dump_counts = d_counts;
  rq.check_status = true;
  rq.stage_timing = h->ws.stage_timing;
  fpp::BatchResult res;
  fpp::Error err{0, ""};
  rc = fpp::batch_query(h->P, h->di, h->bw, rq, s, res, err);
  if (rc) return fail(rc, err.msg);
  if (res.overflow) return fail(FPP_ERR_UNSUPPORTED, "query_batched_dump: candidate capacity exceeded");
  set_batch_stats(h, res);
  return ok();
}

int fpp_query_dump(fpp_index* h, const float* queries, int n_queries, int n_neighbors, int32_t* out,
                   float* topk_val, uint32_t* probes, float* probe_val, long long* stats, int32_t* cands,
                   long long cand_cap) {
  if (!h) return fail(FPP_ERR_INVALID_ARGUMENT, "query_dump: NULL handle");
  std::lock_guard<std::mutex> g(h->mu);
  int rc = check_query_params(h, n_queries, n_neighbors);
  if (rc) return rc;
  if (n_queries > 0 && (!queries || !out)) return fail(FPP_ERR_INVALID_ARGUMENT, "query_dump: NULL buffer");
  if (use_device(h)) return FPP_ERR_CUDA;
  fpp::QueryDumps dumps;
  std::vector<long long> cc(n_queries), uc(n_queries);
  dumps.probes = probes;
  dumps.probe_v = probe_val;
  dumps.topk_v = topk_val;
  dumps.cand_count = cc.data();
  dumps.unique_count = uc.data();
  if (cands && cand_cap < 1) return fail(FPP_ERR_INVALID_ARGUMENT, "query_dump: cand_cap must be >= 1");
  dumps.want_cands = cands != nullptr;
  fpp::Error err{0, ""};
  rc = fpp::query_index(h->P, h->di, queries, false, n_queries, n_neighbors, out, false, h->ws, h->qst, h->stream, err,
                        &dumps);
  if (rc == FPP_OK && cands) {
    for (int q = 0; q < n_queries; ++q) {
      if (uc[q] > cand_cap) return fail(FPP_ERR_INVALID_ARGUMENT, "query_dump: cand_cap smaller than a candidate set");
      for (long long i = 0; i < cand_cap; ++i)
        cands[(size_t)q * cand_cap + i] = i < uc[q] ? dumps.cands[(size_t)q * dumps.cand_stride + i] : -1;
    }
  }
  if (rc) return fail(rc, err.msg);
  if (stats)
    for (int q = 0; q < n_queries; ++q) {
      stats[(size_t)q * 4 + 0] = cc[q];
      stats[(size_t)q * 4 + 1] = uc[q];
      stats[(size_t)q * 4 + 2] = 0;
      stats[(size_t)q * 4 + 3] = h->P.qProbes;
    }
  return ok();
}

int fpp_get_info(fpp_index* h, long long* out, int n) {
  if (!h || !out) return fail(FPP_ERR_INVALID_ARGUMENT, "get_info: NULL argument");
  std::lock_guard<std::mutex> g(h->mu);
  const long long v[9] = {h->P.fhtDim,
                          (long long)h->di.n_ids,
                          (long long)h->di.max_kept,
                          (long long)h->P.n_tables * 4LL * h->P.n_proj * h->P.n_proj,
                          h->built ? 1LL : 0LL,
                          h->device,
                          h->P.n_tables,
                          h->P.n_proj,
                          h->P.iProbes};
  for (int i = 0; i < n && i < 9; ++i) out[i] = v[i];
  return ok();
}

int fpp_get_stats(fpp_index* h, int kind, double* out, int n) {
  if (!h || !out) return fail(FPP_ERR_INVALID_ARGUMENT, "get_stats: NULL argument");
  std::lock_guard<std::mutex> g(h->mu);
  if (kind == 0) {
    const fpp::BuildStats& s = h->bst;
    const double v[8] = {s.ms_center, s.ms_hash, s.ms_sort, s.ms_csr, s.ms_total,
                         (double)s.n_repaired, (double)s.n_limited, s.points_per_table};
    for (int i = 0; i < n && i < 8; ++i) out[i] = v[i];
  } else if (kind == 1) {
    const fpp::QueryStats& s = h->qst;
    const double v[11] = {(double)s.total_cand, (double)s.total_unique, (double)s.total_empty,
                          (double)s.total_probes, (double)s.n_select_ties, (double)s.n_topk_ties,
                          (double)s.launches, s.ms_hash, s.ms_select, s.ms_rerank, (double)s.tc_exact};
    for (int i = 0; i < n && i < 11; ++i) out[i] = v[i];
  } else {
    return fail(FPP_ERR_INVALID_ARGUMENT, "get_stats: kind must be 0 or 1");
  }
  return ok();
}

int fpp_dump_bits(fpp_index* h, uint8_t* b1, uint8_t* b2) {
  if (!h || !b1 || !b2) return fail(FPP_ERR_INVALID_ARGUMENT, "dump_bits: NULL argument");
  std::lock_guard<std::mutex> g(h->mu);
  if (!h->built) return fail(FPP_ERR_NOT_BUILT, "dump_bits: the index is not built");
  memcpy(b1, h->bits.b1.data(), h->bits.b1.size());
  memcpy(b2, h->bits.b2.data(), h->bits.b2.size());
  return ok();
}

int fpp_dump_center(fpp_index* h, float* center) {
  if (!h || !center) return fail(FPP_ERR_INVALID_ARGUMENT, "dump_center: NULL argument");
  std::lock_guard<std::mutex> g(h->mu);
  if (!h->built) return fail(FPP_ERR_NOT_BUILT, "dump_center: the index is not built");
  cudaSetDevice(h->device);
  if (cudaMemcpy(center, h->di.center, sizeof(float) * h->P.n_features, cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(FPP_ERR_CUDA, "dump_center: copy failed");
  return ok();
}

int fpp_dump_tables(fpp_index* h, uint32_t* bucket_start, int32_t* ids) {
  if (!h || !bucket_start || !ids) return fail(FPP_ERR_INVALID_ARGUMENT, "dump_tables: NULL argument");
  std::lock_guard<std::mutex> g(h->mu);
  if (!h->built) return fail(FPP_ERR_NOT_BUILT, "dump_tables: the index is not built");
  cudaSetDevice(h->device);
  const size_t nb = (size_t)h->P.n_tables * 4 * h->P.n_proj * h->P.n_proj + 1;
  if (cudaMemcpy(bucket_start, h->di.bucket_off, sizeof(uint32_t) * nb, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(ids, h->di.ids, sizeof(int32_t) * h->di.n_ids, cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(FPP_ERR_CUDA, "dump_tables: copy failed");
  return ok();
}

void fpp_print_build_report(fpp_index* h) {
  if (!h) return;
  std::lock_guard<std::mutex> g(h->mu);
  print_build(h);
}

}  // extern "C"
