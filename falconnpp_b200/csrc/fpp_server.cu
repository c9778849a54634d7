// fpp_server.cu — continuous-batching serving loop over the batched query form
// (no reference counterpart; the reference answers one synchronous batch per
// call, src/FalconnPP.cpp:310-707).
//
// A worker thread owns S launch slots, one CUDA stream each.  Each slot has
// its own device buffers (queries, per-query k and qProbes, results) and its
// own scratch for the fused kernel, so slots run concurrently on the GPU.
// Requests (1..max_batch queries, their own k and qProbes) wait in a FIFO;
// whenever a slot is free the worker packs the waiting requests into one mixed
// batch — as many as fit the slot and the in-flight memory budget — uploads
// them and launches.  Requests that arrive while other batches run are admitted
// as slots free up, so their work overlaps with the running batches.  A request
// is never split; each query of a batch is answered independently of the
// others, so a request's results do not depend on the batch it lands in.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/falconnpp_b200.h"
#include "fpp_handle.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  long long ticket;
  const float* q;  // host
  int nq, k, qprobes;
  int32_t* out;    // host, nq x k
  Clock::time_point t_submit;
  size_t bytes;
};

struct Done {
  double latency_ms;
  int status;
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  float* dQ = nullptr;
  int32_t* dK = nullptr;
  int32_t* dP = nullptr;
  int32_t* dOut = nullptr;
  float* hQ = nullptr;  // pinned staging
  int32_t* hK = nullptr;
  int32_t* hP = nullptr;
  int32_t* hOut = nullptr;
  fpp::BatchWorkspace bw;
  bool busy = false;
  std::vector<Request> reqs;
  int nq = 0;
};

}  // namespace

struct fpp_server {
  fpp_index* h = nullptr;
  int max_batch = 0, k_max = 0, qprobes_max = 0;
  size_t budget = 0, inflight = 0;
  std::vector<Slot> slots;
  std::deque<Request> pending;
  std::map<long long, Done> done;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  long long next_ticket = 1;
  long long launches = 0, queries = 0, requests = 0;
  std::thread worker;
  int device = 0;
};

namespace {

size_t request_bytes(int nq, int d, int k) { return (size_t)nq * ((size_t)d * 4 + (size_t)k * 4 + 8); }

void free_slot(Slot& s) {
  if (s.stream) cudaStreamSynchronize(s.stream);
  cudaFree(s.dQ);
  cudaFree(s.dK);
  cudaFree(s.dP);
  cudaFree(s.dOut);
  cudaFreeHost(s.hQ);
  cudaFreeHost(s.hK);
  cudaFreeHost(s.hP);
  cudaFreeHost(s.hOut);
  s.bw.release();
  if (s.done) cudaEventDestroy(s.done);
  if (s.stream) cudaStreamDestroy(s.stream);
}

// Completes a finished slot: copies each request's rows to its host buffer.
void finish_slot(fpp_server* S, Slot& s, int status) {
  const int kmax = S->k_max;
  int row = 0;
  const auto now = Clock::now();
  for (const Request& r : s.reqs) {
    if (status == FPP_OK)
      for (int i = 0; i < r.nq; ++i)
        memcpy(r.out + (size_t)i * r.k, s.hOut + (size_t)(row + i) * kmax, sizeof(int32_t) * r.k);
    row += r.nq;
    S->done[r.ticket] = Done{std::chrono::duration<double, std::milli>(now - r.t_submit).count(), status};
    S->inflight -= r.bytes;
  }
  s.reqs.clear();
  s.busy = false;
  s.nq = 0;
}

// the batch request of slot s for nq staged queries (per-query k and qProbes
// in dK / dP)
fpp::BatchRequest slot_request(const fpp_server* S, const Slot& s, int nq) {
  const fpp_index* h = S->h;
  fpp::BatchRequest rq;
  rq.Q = s.dQ;
  rq.nq = nq;
  rq.q_k = s.dK;
  rq.q_qprobes = s.dP;
  rq.k_uniform = S->k_max;
  rq.qprobes_uniform = S->qprobes_max;
  rq.k_max = S->k_max;
  rq.qprobes_max = S->qprobes_max;
  rq.mode = h->precision;
  rq.shortlist_mult = h->shortlist_mult;
  rq.out = s.dOut;
  rq.out_stride = S->k_max;
  rq.check_status = false;
  rq.blocks_per_sm = std::max(1, 3 / (int)S->slots.size());
  rq.reorder = h->reorder;
  rq.tc_rotation = h->tc_rotation;
  rq.split_hash = h->split_hash;
  rq.tc_hash = h->tc_hash;
  return rq;
}

void worker_loop(fpp_server* S) {
  cudaSetDevice(S->device);
  const fpp_index* h = S->h;
  const int d = h->P.n_features;
  std::unique_lock<std::mutex> lk(S->mu);
  for (;;) {
    // retire finished slots
    bool progressed = false;
    for (Slot& s : S->slots) {
      if (!s.busy) continue;
      const cudaError_t q = cudaEventQuery(s.done);
      if (q == cudaErrorNotReady) continue;
      finish_slot(S, s, q == cudaSuccess ? FPP_OK : FPP_ERR_CUDA);
      progressed = true;
    }
    if (progressed) S->cv_done.notify_all();
    // admit waiting requests into free slots
    for (Slot& s : S->slots) {
      if (s.busy || S->pending.empty()) continue;
      int nq = 0;
      while (!S->pending.empty()) {
        const Request& r = S->pending.front();
        if (nq + r.nq > S->max_batch) break;
        if (nq > 0 && S->inflight + r.bytes > S->budget) break;  // memory gate
        s.reqs.push_back(r);
        S->inflight += r.bytes;
        nq += r.nq;
        S->pending.pop_front();
      }
      if (nq == 0) continue;
      int row = 0;
      for (const Request& r : s.reqs) {  // stage queries, per-query k and qProbes
        memcpy(s.hQ + (size_t)row * d, r.q, sizeof(float) * (size_t)r.nq * d);
        for (int i = 0; i < r.nq; ++i) {
          s.hK[row + i] = r.k;
          s.hP[row + i] = r.qprobes;
        }
        row += r.nq;
      }
      s.nq = nq;
      s.busy = true;
      S->launches++;
      S->queries += nq;
      lk.unlock();
      cudaMemcpyAsync(s.dQ, s.hQ, sizeof(float) * (size_t)nq * d, cudaMemcpyHostToDevice, s.stream);
      cudaMemcpyAsync(s.dK, s.hK, sizeof(int32_t) * nq, cudaMemcpyHostToDevice, s.stream);
      cudaMemcpyAsync(s.dP, s.hP, sizeof(int32_t) * nq, cudaMemcpyHostToDevice, s.stream);
      const fpp::BatchRequest rq = slot_request(S, s, nq);
      fpp::BatchResult res;
      fpp::Error err{0, ""};
      const int rc = fpp::batch_query(h->P, const_cast<fpp::DeviceIndex&>(h->di), s.bw, rq, s.stream, res, err);
      if (rc == FPP_OK) {
        cudaMemcpyAsync(s.hOut, s.dOut, sizeof(int32_t) * (size_t)nq * S->k_max, cudaMemcpyDeviceToHost, s.stream);
        cudaEventRecord(s.done, s.stream);
      }
      lk.lock();
      if (rc != FPP_OK) {
        finish_slot(S, s, rc);
        S->cv_done.notify_all();
      }
    }
    bool any_busy = false;
    for (const Slot& s : S->slots) any_busy |= s.busy;
    if (S->stop && !any_busy && S->pending.empty()) break;
    if (any_busy) {
      S->cv_work.wait_for(lk, std::chrono::microseconds(20));  // poll the running batches
    } else {
      S->cv_work.wait(lk, [S] { return S->stop || !S->pending.empty(); });
    }
  }
}

}  // namespace

extern "C" {

int fpp_server_create(fpp_index* h, int n_streams, long long memory_budget_bytes, int max_batch, int k_max,
                      int qprobes_max, fpp_server** out) {
  if (!h || !out) return fpp::set_last_error(FPP_ERR_INVALID_ARGUMENT, "server_create: NULL argument");
  *out = nullptr;
  if (!h->built) return fpp::set_last_error(FPP_ERR_NOT_BUILT, "server_create: the index is not built");
  if (n_streams < 1 || n_streams > 8 || max_batch < 1 || k_max < 1 || k_max > 1024 || qprobes_max < 1 ||
      memory_budget_bytes <= 0)
    return fpp::set_last_error(FPP_ERR_INVALID_ARGUMENT,
                               "server_create: need 1..8 streams, max_batch >= 1, 1 <= k_max <= 1024, "
                               "qprobes_max >= 1, a positive memory budget");
  cudaSetDevice(h->device);
  if (h->precision != 0) {
    fpp::Error err{0, ""};
    const int rc = fpp::ensure_lowp_rows(h->P, h->di, h->precision, h->stream, err);
    if (rc) return fpp::set_last_error(rc, err.msg);
  }
  fpp_server* S = new fpp_server();
  S->h = h;
  S->device = h->device;
  S->max_batch = max_batch;
  S->k_max = k_max;
  S->qprobes_max = qprobes_max;
  S->budget = (size_t)memory_budget_bytes;
  S->slots.resize(n_streams);
  const int d = h->P.n_features;
  bool ok = true;
  for (Slot& s : S->slots) {
    ok = ok && cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming) == cudaSuccess;
    ok = ok && fpp::dev_malloc(&s.dQ, sizeof(float) * (size_t)max_batch * d) == cudaSuccess;
    ok = ok && fpp::dev_malloc(&s.dK, sizeof(int32_t) * max_batch) == cudaSuccess;
    ok = ok && fpp::dev_malloc(&s.dP, sizeof(int32_t) * max_batch) == cudaSuccess;
    ok = ok && fpp::dev_malloc(&s.dOut, sizeof(int32_t) * (size_t)max_batch * k_max) == cudaSuccess;
    ok = ok && cudaMallocHost(&s.hQ, sizeof(float) * (size_t)max_batch * d) == cudaSuccess;
    ok = ok && cudaMallocHost(&s.hK, sizeof(int32_t) * max_batch) == cudaSuccess;
    ok = ok && cudaMallocHost(&s.hP, sizeof(int32_t) * max_batch) == cudaSuccess;
    ok = ok && cudaMallocHost(&s.hOut, sizeof(int32_t) * (size_t)max_batch * k_max) == cudaSuccess;
    if (!ok) break;
  }
  if (!ok) {
    for (Slot& s : S->slots) free_slot(s);
    delete S;
    return fpp::set_last_error(FPP_ERR_OUT_OF_MEMORY, "server_create: cannot allocate the slots");
  }
  // Warm-up: one batch of max_batch zero queries at k_max and qprobes_max
  // per slot sizes the slot's batch workspace (per-block scratch, query-order
  // buffers) for the largest batch a request mix can form, and loads the
  // kernel.  Without it the first batches allocate while others run, and a
  // workspace that grows frees its old buffers, which waits for the whole
  // device: the requests in flight on every stream would see the stall.
  for (Slot& s : S->slots) {
    for (int i = 0; i < max_batch; ++i) {
      s.hK[i] = k_max;
      s.hP[i] = qprobes_max;
    }
    ok = ok && cudaMemsetAsync(s.dQ, 0, sizeof(float) * (size_t)max_batch * d, s.stream) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(s.dK, s.hK, sizeof(int32_t) * max_batch, cudaMemcpyHostToDevice, s.stream) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(s.dP, s.hP, sizeof(int32_t) * max_batch, cudaMemcpyHostToDevice, s.stream) == cudaSuccess;
    if (!ok) break;
    const fpp::BatchRequest rq = slot_request(S, s, max_batch);
    fpp::BatchResult res;
    fpp::Error err{0, ""};
    const int rc = fpp::batch_query(h->P, h->di, s.bw, rq, s.stream, res, err);
    if (rc != FPP_OK || cudaStreamSynchronize(s.stream) != cudaSuccess) {
      for (Slot& t : S->slots) free_slot(t);
      delete S;
      return fpp::set_last_error(rc != FPP_OK ? rc : FPP_ERR_CUDA,
                                 std::string("server_create: warm-up batch: ") + err.msg);
    }
  }
  if (!ok) {
    for (Slot& s : S->slots) free_slot(s);
    delete S;
    return fpp::set_last_error(FPP_ERR_CUDA, "server_create: warm-up staging failed");
  }
  S->worker = std::thread(worker_loop, S);
  *out = S;
  return fpp::clear_last_error();
}

int fpp_server_submit(fpp_server* S, const float* queries, int n_queries, int k, int qprobes, int32_t* out,
                      long long* ticket) {
  if (!S || !queries || !out || !ticket) return fpp::set_last_error(FPP_ERR_INVALID_ARGUMENT, "server_submit: NULL");
  if (n_queries < 1 || n_queries > S->max_batch || k < 1 || k > S->k_max || qprobes < 1 || qprobes > S->qprobes_max)
    return fpp::set_last_error(FPP_ERR_INVALID_ARGUMENT,
                               "server_submit: need 1 <= n_queries <= max_batch, 1 <= k <= k_max, "
                               "1 <= qProbes <= qprobes_max");
  Request r;
  r.q = queries;
  r.nq = n_queries;
  r.k = k;
  r.qprobes = qprobes;
  r.out = out;
  r.t_submit = Clock::now();
  r.bytes = request_bytes(n_queries, S->h->P.n_features, S->k_max);
  {
    std::lock_guard<std::mutex> g(S->mu);
    if (S->stop) return fpp::set_last_error(FPP_ERR_INVALID_ARGUMENT, "server_submit: server is stopping");
    r.ticket = S->next_ticket++;
    S->requests++;
    S->pending.push_back(r);
    *ticket = r.ticket;
  }
  S->cv_work.notify_one();
  return fpp::clear_last_error();
}

int fpp_server_wait(fpp_server* S, long long ticket, double* latency_ms) {
  if (!S) return fpp::set_last_error(FPP_ERR_INVALID_ARGUMENT, "server_wait: NULL");
  std::unique_lock<std::mutex> lk(S->mu);
  if (ticket < 1 || ticket >= S->next_ticket)
    return fpp::set_last_error(FPP_ERR_INVALID_ARGUMENT, "server_wait: bad ticket");
  S->cv_done.wait(lk, [&] { return S->done.count(ticket) > 0; });
  const Done d = S->done[ticket];
  S->done.erase(ticket);
  if (latency_ms) *latency_ms = d.latency_ms;
  if (d.status != FPP_OK) return fpp::set_last_error(d.status, "server: the batch holding this request failed");
  return fpp::clear_last_error();
}

int fpp_server_stats(fpp_server* S, double* out, int n) {
  if (!S || !out) return fpp::set_last_error(FPP_ERR_INVALID_ARGUMENT, "server_stats: NULL");
  std::lock_guard<std::mutex> g(S->mu);
  const double v[4] = {(double)S->launches, (double)S->queries, (double)S->requests, (double)S->pending.size()};
  for (int i = 0; i < n && i < 4; ++i) out[i] = v[i];
  return fpp::clear_last_error();
}

void fpp_server_destroy(fpp_server* S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> g(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  if (S->worker.joinable()) S->worker.join();
  cudaSetDevice(S->device);
  for (Slot& s : S->slots) free_slot(s);
  delete S;
}

}  // extern "C"
