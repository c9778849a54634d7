// fpp_batch.cu — the batched query form: ONE persistent kernel per batch that
// runs rotate -> hash -> probe selection -> gather/dedupe -> rerank -> top-k for
// every query (src/FalconnPP.cpp:345-677 per query), with
//
//   * dynamic scheduling: blocks take queries from a work counter, so uneven
//     qProbes and candidate counts balance across the GPU;
//   * per-query k and qProbes (arrays), for mixed batches;
//   * reranking of the candidate rows in BF16 or FP8-E4M3 (per-row FP32 scale)
//     with FP32 accumulation, then an exact FP32 re-score of a shortlist of
//     r*k candidates and the top-k of the shortlist; in FP32 mode the kernel
//     reproduces the plain path bit for bit;
//   * optional capture of the launch (work-counter reset + kernel) in a CUDA
//     graph; later calls with the same grid replay it, updating the kernel
//     node's arguments (batch size, buffers, k, qProbes) in place.
//
// Hashing, probe selection and the tie rules are the plain path's
// (fpp_query.cu): the hash arithmetic stays FP32 and bit-exact.
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <vector>

#include "fpp_batch_kernel.cuh"
#include "fpp_query.h"

namespace fpp {

// ---------------------------------------------------------------- conversion
__global__ void k_rows_bf16(const float* __restrict__ Xc, long long n, int ld, int ldo, uint16_t* __restrict__ out) {
  const long long total = n * (long long)ldo;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const long long i = t / ldo;
    const int j = (int)(t - i * ldo);
    const float x = j < ld ? Xc[i * ld + j] : 0.0f;
    const __nv_bfloat16 b = __float2bfloat16_rn(x);
    out[t] = *reinterpret_cast<const uint16_t*>(&b);
  }
}

// one warp per row: scale = max|x| / 448 (E4M3 largest finite), x8 = x / scale
__global__ void k_rows_fp8(const float* __restrict__ Xc, long long n, int ld, int ldo, uint8_t* __restrict__ out,
                           float* __restrict__ scale) {
  const int lane = threadIdx.x & 31;
  const long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long i = w; i < n; i += nw) {
    float mx = 0.0f;
    for (int j = lane; j < ld; j += 32) mx = fmaxf(mx, fabsf(Xc[i * ld + j]));
    for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    const float s = mx > 0.0f ? mx / 448.0f : 1.0f;
    for (int j = lane; j < ldo; j += 32) {
      const float x = j < ld ? Xc[i * ld + j] / s : 0.0f;
      out[i * ldo + j] = (uint8_t)__nv_cvt_float_to_fp8(x, __NV_SATFINITE, __NV_E4M3);
    }
    if (lane == 0) scale[i] = s;
  }
}

// ---------------------------------------------------------------- query order
// A batch is processed grouped by each query's best bucket code in layer 0 of
// table 0 (the cross-polytope code of its largest rotated coordinate): the
// queries in flight at the same time then probe overlapping buckets and rows,
// which stay in L2.  Each query is computed independently, so the order
// changes no result.
constexpr int kOrderMaxBins = 1024;  // 2 * n_proj codes

template <int FHT>
__global__ void __launch_bounds__(256) k_order_key(const float* __restrict__ Q, int nq, int d,
                                                   const uint32_t* __restrict__ flips, int D, int log2D,
                                                   uint32_t* __restrict__ key, uint32_t* __restrict__ hist) {
  constexpr int E = Geo<FHT>::E;
  constexpr int G = Geo<FHT>::G;
  const int gl = threadIdx.x & (G - 1);
  const long long q = (long long)blockIdx.x * (blockDim.x / G) + threadIdx.x / G;
  const bool active = q < nq;  // inactive groups still join every shuffle
  float y[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int idx = gl * E + e;
    y[e] = (active && idx < d) ? __ldg(Q + (size_t)q * d + idx) : 0.0f;
  }
  hd3_rotate<FHT>(y, flips, gl);  // (layer 0, table 0) flips come first
  float v = 0.0f;
  int c = 0;
  group_top2_cp<FHT>(y, gl, D, log2D, 1, &v, &c);
  if (gl == 0 && active) {
    key[q] = (uint32_t)c;
    atomicAdd(hist + c, 1u);
  }
}

// one block of 1024 threads: counting sort of the keys into `order`; leaves
// the histogram zeroed for the next batch
__global__ void __launch_bounds__(1024) k_order_scatter(const uint32_t* __restrict__ key, int nq, int bins,
                                                        uint32_t* __restrict__ hist, uint32_t* __restrict__ order) {
  __shared__ uint32_t off[kOrderMaxBins];
  __shared__ long long tmp[32];
  const int t = threadIdx.x;
  const uint32_t h = t < bins ? hist[t] : 0u;
  long long tot;
  const long long ex = block_exclusive_scan((long long)h, tmp, &tot);
  if (t < bins) {
    off[t] = (uint32_t)ex;
    hist[t] = 0u;
  }
  __syncthreads();
  for (int q = t; q < nq; q += blockDim.x) order[atomicAdd(&off[key[q]], 1u)] = (uint32_t)q;
}

// the key from the exact lists: the first-layer code of table 0's best bucket
__global__ void k_order_key_ext(const uint32_t* __restrict__ lb, int nq, long long stride, int twoD,
                                uint32_t* __restrict__ key, uint32_t* __restrict__ hist) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nq) return;
  const uint32_t c = lb[(size_t)q * stride] / (uint32_t)twoD;  // table 0: global id = c1 * 2D + c2
  key[q] = c;
  atomicAdd(hist + c, 1u);
}

static const void* order_key_kernel(int fht) {
  switch (fht) {
    case 32: return reinterpret_cast<const void*>(&k_order_key<32>);
    case 64: return reinterpret_cast<const void*>(&k_order_key<64>);
    case 128: return reinterpret_cast<const void*>(&k_order_key<128>);
    case 256: return reinterpret_cast<const void*>(&k_order_key<256>);
    case 512: return reinterpret_cast<const void*>(&k_order_key<512>);
    default: return nullptr;
  }
}

// ---------------------------------------------------------------- host side
int ensure_lowp_rows(const Params& P, DeviceIndex& di, int mode, cudaStream_t s, Error& err) {
  if (mode == kRowsF32 || di.lp_mode == mode) return kOk;
  cudaFree(di.Xlp);
  cudaFree(di.Xlp_scale);
  di.Xlp = nullptr;
  di.Xlp_scale = nullptr;
  di.lp_mode = kRowsF32;
  const long long n = P.n_points;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaError_t e;
  if (mode == kRowsBF16) {
    const int ldo = (P.n_features + 7) & ~7;  // 16-byte rows
    if ((e = fpp::dev_malloc(&di.Xlp, (size_t)n * ldo * 2)) != cudaSuccess) goto fail;
    k_rows_bf16<<<nsm * 8, 256, 0, s>>>(di.Xc, n, di.ld, ldo, static_cast<uint16_t*>(di.Xlp));
    di.ld_lp = ldo;
  } else {
    const int ldo = (P.n_features + 15) & ~15;
    if ((e = fpp::dev_malloc(&di.Xlp, (size_t)n * ldo)) != cudaSuccess) goto fail;
    if ((e = fpp::dev_malloc(&di.Xlp_scale, sizeof(float) * n)) != cudaSuccess) goto fail;
    k_rows_fp8<<<nsm * 8, 256, 0, s>>>(di.Xc, n, di.ld, ldo, static_cast<uint8_t*>(di.Xlp), di.Xlp_scale);
    di.ld_lp = ldo;
  }
  if ((e = cudaGetLastError()) != cudaSuccess) goto fail;
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) goto fail;
  di.lp_mode = mode;
  return kOk;
fail:
  err.code = (e == cudaErrorMemoryAllocation) ? kErrOutOfMemory : kErrCuda;
  err.msg = std::string("low-precision rows: ") + cudaGetErrorString(e);
  cudaFree(di.Xlp);
  cudaFree(di.Xlp_scale);
  di.Xlp = nullptr;
  di.Xlp_scale = nullptr;
  return err.code;
}

void BatchWorkspace::release() {
  if (graph_exec) cudaGraphExecDestroy(graph_exec);
  if (graph) cudaGraphDestroy(graph);
  cudaFree(bitset);
  cudaFree(uniq);
  cudaFree(score);
  cudaFree(gdump);
  cudaFree(gheap_v);
  cudaFree(gheap_i);
  cudaFree(counters);
  for (auto& ev : tev)
    if (ev) cudaEventDestroy(ev);
  for (auto& ev : cev)
    if (ev) cudaEventDestroy(ev);
  cudaFree(okey);
  cudaFree(ohist);
  cudaFree(order);
  cudaFree(glv);
  cudaFree(glb);
  cudaFree(gprobe);
  cudaFree(gpo);
  cudaFree(gpe);
  cudaFree(ggv);
  cudaFree(ggc);
  cudaFree(grhv);
  cudaFree(grhi);
  cudaFree(ext_lv);
  cudaFree(ext_lb);
  cudaFree(hheap_v);
  cudaFree(hheap_i);
  cudaFree(pc_g);
  cudaFree(pc_o);
  cudaFree(pc_pe);
  cudaFree(pc_n);
  *this = BatchWorkspace();
}

static KernelSel pick_kernel(int fht, int mode, int d, bool tc_only) {
  if (d > 512) return KernelSel{nullptr, 0};
  if (mode == kRowsF32) return pick_kernel_f32(fht, d);
  if (mode == kRowsBF16) return pick_kernel_bf16(fht, d, tc_only);
  return pick_kernel_fp8(fht, d, tc_only);
}

int batch_query(const Params& P, DeviceIndex& di, BatchWorkspace& bw, const BatchRequest& rq, cudaStream_t s,
                BatchResult& res, Error& err) {
  auto fail = [&](cudaError_t e, const char* what) {
    err.code = (e == cudaErrorMemoryAllocation) ? kErrOutOfMemory : kErrCuda;
    err.msg = std::string("batch query: ") + what + ": " + cudaGetErrorString(e);
    return err.code;
  };
  res = BatchResult();
  if (rq.nq <= 0) return kOk;
  const int L = P.n_tables, D = P.n_proj, d = P.n_features, F = P.fhtDim;
  const int mmax = (2 * rq.qprobes_max + L - 1) / L;
  int m1max = 0;
  while (m1max * m1max < mmax) ++m1max;
  // lists, probes and prefixes beyond the shared-memory capacities: the
  // big-list instances keep them in per-block global scratch
  const bool big = rq.qprobes_max > kBMaxProbes || (long long)L * mmax > kBMaxList || m1max > kBMaxM1;
  if (m1max > kBigM1 || m1max > D || L > kBigMaxL || (long long)L * mmax > (1LL << 24)) {
    err.code = kErrUnsupported;
    err.msg = "batch query: outside the batched form's limits (ceil(sqrt(ceil(2 qProbes / n_tables))) <= "
              "min(32, n_proj), n_tables <= 512); use the plain form";
    return err.code;
  }
  if (rq.k_max < 1 || (long long)rq.k_max * (rq.mode == kRowsF32 ? 1 : rq.shortlist_mult) > kBMaxTop) {
    err.code = kErrInvalidArgument;
    err.msg = "batch query: k * shortlist multiple must be <= 1024";
    return err.code;
  }
  if (rq.mode != kRowsF32) {
    const int rc = ensure_lowp_rows(P, di, rq.mode, s, err);
    if (rc) return rc;
  }
  // every query keeps one probe per table (2 qProbes <= L): the kernel
  // without the exact rotation
  const bool tc_only =
      !big && rq.tc_rotation && rq.mode != kRowsF32 && F == 256 && di.tflips && 2 * rq.qprobes_max <= L;
  // the exact hash in its own kernel (k_query_hash with per-query qProbes),
  // then the fused kernel without the rotation compiled in
  const bool split = rq.split_hash && !tc_only && d <= 512;
  const KernelSel ks = split ? pick_kernel_ext(rq.mode, d, big)
                       : big ? (d > 512 ? KernelSel{nullptr, 0} : pick_kernel_big(F, rq.mode, d))
                             : pick_kernel(F, rq.mode, d, tc_only);
  const void* kern = ks.fn;
  if (!kern) {
    err.code = kErrUnsupported;
    err.msg = "batch query: the batched form covers fhtDim 32..512 and d <= 512; use the plain form";
    return err.code;
  }
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaError_t e;
  int per_sm = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBThreads, ks.smem)) != cudaSuccess)
    return fail(e, "occupancy");
  if (rq.blocks_per_sm > 0) per_sm = std::min(per_sm, rq.blocks_per_sm);
  per_sm = std::max(per_sm, 1);
  // graph mode keeps one grid for every batch size (idle blocks find no work)
  int grid = std::max(1, rq.use_graph ? nsm * per_sm : std::min(rq.nq, nsm * per_sm));
  const long long nwords = (P.n_points + 31) / 32;
  const long long cap = std::max<long long>(
      1, std::min<long long>(P.n_points, (long long)rq.qprobes_max * std::max<uint32_t>(di.max_kept, 1u)));
  const int groups = grid * (kBThreads / (F < 32 ? 1 : F / 32));
  const long long list_cap = big ? (long long)L * mmax : 0;
  const long long probe_cap = big ? rq.qprobes_max : 0;
  // (re)allocate per-block scratch when the shape grows
  if (!bw.bitset || bw.grid < grid || bw.nwords != nwords || bw.cap < cap || bw.fht < F || bw.mmax < mmax ||
      bw.list_cap < list_cap || bw.probe_cap < probe_cap) {
    bw.release();
    if ((e = fpp::dev_malloc(&bw.bitset, sizeof(uint32_t) * (size_t)grid * nwords)) != cudaSuccess) return fail(e, "alloc");
    if ((e = cudaMemsetAsync(bw.bitset, 0, sizeof(uint32_t) * (size_t)grid * nwords, s)) != cudaSuccess)
      return fail(e, "memset");
    if ((e = fpp::dev_malloc(&bw.uniq, sizeof(uint32_t) * (size_t)grid * cap)) != cudaSuccess) return fail(e, "alloc");
    if ((e = fpp::dev_malloc(&bw.score, sizeof(uint32_t) * (size_t)grid * cap)) != cudaSuccess) return fail(e, "alloc");
    if ((e = fpp::dev_malloc(&bw.gdump, sizeof(float) * (size_t)groups * F)) != cudaSuccess) return fail(e, "alloc");
    if ((e = fpp::dev_malloc(&bw.gheap_v, sizeof(float) * (size_t)groups * std::max(mmax, 1))) != cudaSuccess)
      return fail(e, "alloc");
    if ((e = fpp::dev_malloc(&bw.gheap_i, sizeof(int) * (size_t)groups * std::max(mmax, 1))) != cudaSuccess)
      return fail(e, "alloc");
    if ((e = fpp::dev_malloc(&bw.counters, sizeof(unsigned) * 4)) != cudaSuccess) return fail(e, "alloc");
    if (big) {
      const size_t gl = (size_t)grid * list_cap, gp = (size_t)grid * probe_cap;
      const size_t gg = (size_t)groups * 2 * (kBigM1 + 1), gr = (size_t)groups * kBigM1;
      if ((e = fpp::dev_malloc(&bw.glv, sizeof(float) * gl)) != cudaSuccess ||
          (e = fpp::dev_malloc(&bw.glb, sizeof(uint32_t) * gl)) != cudaSuccess ||
          (e = fpp::dev_malloc(&bw.gprobe, sizeof(uint32_t) * gp)) != cudaSuccess ||
          (e = fpp::dev_malloc(&bw.gpo, sizeof(uint32_t) * gp)) != cudaSuccess ||
          (e = fpp::dev_malloc(&bw.gpe, sizeof(uint32_t) * gp)) != cudaSuccess ||
          (e = fpp::dev_malloc(&bw.ggv, sizeof(float) * gg)) != cudaSuccess ||
          (e = fpp::dev_malloc(&bw.ggc, sizeof(int) * gg)) != cudaSuccess ||
          (e = fpp::dev_malloc(&bw.grhv, sizeof(float) * gr)) != cudaSuccess ||
          (e = fpp::dev_malloc(&bw.grhi, sizeof(int) * gr)) != cudaSuccess)
        return fail(e, "alloc");
    }
    bw.list_cap = list_cap;
    bw.probe_cap = probe_cap;
    bw.grid = grid;
    bw.nwords = nwords;
    bw.cap = cap;
    bw.fht = F;
    bw.mmax = std::max(mmax, 1);
  }
  grid = std::min(grid, bw.grid);
  const long long ext_stride = (long long)L * std::max(mmax, 1);
  const bool vhash = split && rq.tc_hash && F == 256 && di.tflips && L <= 128 && 2 * rq.qprobes_max <= L;
  if (split) {
    const long long max_groups = (long long)nsm * 64;
    if (!bw.ext_lv || bw.ext_cap < (long long)rq.nq * ext_stride) {
      cudaFree(bw.ext_lv);
      cudaFree(bw.ext_lb);
      bw.ext_lv = nullptr;
      bw.ext_lb = nullptr;
      bw.ext_cap = 0;
      const size_t ne = (size_t)rq.nq * ext_stride;
      if ((e = fpp::dev_malloc(&bw.ext_lv, sizeof(float) * ne)) != cudaSuccess ||
          (e = fpp::dev_malloc(&bw.ext_lb, sizeof(uint32_t) * ne)) != cudaSuccess)
        return fail(e, "alloc");
      bw.ext_cap = (long long)ne;
    }
    if (!bw.hheap_v || bw.hheap_cap < max_groups * std::max(mmax, 1)) {
      cudaFree(bw.hheap_v);
      cudaFree(bw.hheap_i);
      bw.hheap_v = nullptr;
      bw.hheap_i = nullptr;
      bw.hheap_cap = 0;
      const size_t nh = (size_t)max_groups * std::max(mmax, 1);
      if ((e = fpp::dev_malloc(&bw.hheap_v, sizeof(float) * nh)) != cudaSuccess ||
          (e = fpp::dev_malloc(&bw.hheap_i, sizeof(int) * nh)) != cudaSuccess)
        return fail(e, "alloc");
      bw.hheap_cap = (long long)nh;
    }
    if (rq.stage_timing) {
      for (auto& ev : bw.tev)
        if (!ev && (e = cudaEventCreate(&ev)) != cudaSuccess) return fail(e, "event create");
      if (vhash && (e = cudaMemsetAsync(bw.counters + 2, 0, sizeof(unsigned), s)) != cudaSuccess)
        return fail(e, "memset");
      cudaEventRecord(bw.tev[0], s);
    }
    // host queries: up to four chunks copied on the copy stream, each hashed
    // as soon as it lands.  The hash launches of one stream run one after
    // the other, so a chunk that is not a whole number of waves of hash
    // blocks leaves SMs idle at its end: with the verified hash the first
    // chunks are one full wave each and the last takes the rest (the same
    // number of waves as one launch over the batch); otherwise quarters.
    long long cut[5] = {0, 0, 0, 0, 0};
    int nch = (rq.Q_host && rq.copy_stream && rq.copy_stream != s && rq.nq >= 4096) ? 4 : 1;
    if (nch > 1) {
      const long long wq = vhash ? hash_verified_wave_queries() : 0;
      if (wq > 0) nch = (int)std::min<long long>(4, rq.nq / wq);
      for (int c = 0; c <= nch; ++c) cut[c] = wq > 0 ? (c < nch ? c * wq : rq.nq) : (long long)rq.nq * c / nch;
    }
    if (nch <= 1) {
      nch = 1;
      cut[0] = 0;
      cut[1] = rq.nq;
    }
    if (rq.Q_host && nch == 1 &&
        (e = cudaMemcpyAsync(const_cast<float*>(rq.Q), rq.Q_host, sizeof(float) * (size_t)rq.nq * d,
                             cudaMemcpyHostToDevice, s)) != cudaSuccess)
      return fail(e, "query copy");
    if (nch > 1) {
      for (auto& ev : bw.cev)
        if (!ev && (e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess)
          return fail(e, "event create");
      // the copies wait for the stream's earlier work (a previous batch may
      // still read the query buffer)
      cudaEventRecord(bw.cev[4], s);
      cudaStreamWaitEvent(rq.copy_stream, bw.cev[4], 0);
      for (int c = 0; c < nch; ++c) {
        const long long q0 = cut[c], q1 = cut[c + 1];
        if ((e = cudaMemcpyAsync(const_cast<float*>(rq.Q) + q0 * d, rq.Q_host + q0 * d,
                                 sizeof(float) * (size_t)(q1 - q0) * d, cudaMemcpyHostToDevice, rq.copy_stream)) !=
            cudaSuccess)
          return fail(e, "query copy");
        cudaEventRecord(bw.cev[c], rq.copy_stream);
      }
    }
    for (int c = 0; c < nch; ++c) {
      const long long q0 = cut[c], q1 = cut[c + 1];
      if (nch > 1) cudaStreamWaitEvent(s, bw.cev[c], 0);
      const int* qq = rq.q_qprobes ? rq.q_qprobes + q0 : nullptr;
      e = vhash ? hash_lists_verified(P, di, rq.Q + q0 * d, (int)(q1 - q0), qq, rq.qprobes_max,
                                      bw.ext_lv + q0 * ext_stride, bw.ext_lb + q0 * ext_stride, ext_stride,
                                      rq.stage_timing ? bw.counters + 2 : nullptr, s)
                : hash_lists(P, di, rq.Q + q0 * d, (int)(q1 - q0), qq, rq.qprobes_max, bw.ext_lv + q0 * ext_stride,
                             bw.ext_lb + q0 * ext_stride, ext_stride, bw.hheap_v, bw.hheap_i, max_groups, s);
      if (e != cudaSuccess) return fail(e, "hash kernel");
    }
    if (rq.stage_timing) cudaEventRecord(bw.tev[3], s);
  } else if (rq.Q_host) {
    if ((e = cudaMemcpyAsync(const_cast<float*>(rq.Q), rq.Q_host, sizeof(float) * (size_t)rq.nq * d,
                             cudaMemcpyHostToDevice, s)) != cudaSuccess)
      return fail(e, "query copy");
  }
  // query order (worth it once the batch is a few waves of blocks)
  int log2D = 0;
  while ((1 << log2D) < D) ++log2D;
  const void* okern = order_key_kernel(F);
  const bool reorder = rq.reorder && okern && rq.nq >= 2 * grid && 2 * D <= kOrderMaxBins;
  if (reorder && bw.order_cap < rq.nq) {
    cudaFree(bw.okey);
    cudaFree(bw.ohist);
    cudaFree(bw.order);
    bw.okey = bw.ohist = bw.order = nullptr;
    bw.order_cap = 0;
    if ((e = fpp::dev_malloc(&bw.okey, sizeof(uint32_t) * (size_t)rq.nq)) != cudaSuccess) return fail(e, "alloc");
    if ((e = fpp::dev_malloc(&bw.order, sizeof(uint32_t) * (size_t)rq.nq)) != cudaSuccess) return fail(e, "alloc");
    if ((e = fpp::dev_malloc(&bw.ohist, sizeof(uint32_t) * kOrderMaxBins)) != cudaSuccess) return fail(e, "alloc");
    if ((e = cudaMemsetAsync(bw.ohist, 0, sizeof(uint32_t) * kOrderMaxBins, s)) != cudaSuccess)
      return fail(e, "memset");
    bw.order_cap = rq.nq;
  }
  if (reorder && split) {
    k_order_key_ext<<<(rq.nq + 255) / 256, 256, 0, s>>>(bw.ext_lb, rq.nq, ext_stride, 2 * D, bw.okey, bw.ohist);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "order key launch");
    k_order_scatter<<<1, 1024, 0, s>>>(bw.okey, rq.nq, 2 * D, bw.ohist, bw.order);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "order scatter launch");
  } else if (reorder) {
    const int per_block = 256 / (F / 32);
    const float* q_ptr = rq.Q;
    int nq_arg = rq.nq, d_arg = d, D_arg = D, l2_arg = log2D, bins = 2 * D;
    const uint32_t* fl = di.flips;
    void* kargs[] = {&q_ptr, &nq_arg, &d_arg, &fl, &D_arg, &l2_arg, &bw.okey, &bw.ohist};
    if ((e = cudaLaunchKernel(okern, dim3((rq.nq + per_block - 1) / per_block), dim3(256), kargs, 0, s)) !=
        cudaSuccess)
      return fail(e, "order key launch");
    k_order_scatter<<<1, 1024, 0, s>>>(bw.okey, rq.nq, bins, bw.ohist, bw.order);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "order scatter launch");
  }
  // split hash, small lists: the probe cut of every query in its own kernel
  const bool pcut = split && !big;
  if (pcut) {
    const long long npc = (long long)rq.nq * rq.qprobes_max;
    if (!bw.pc_g || bw.pc_cap < npc || bw.pc_ncap < rq.nq) {
      cudaFree(bw.pc_g);
      cudaFree(bw.pc_o);
      cudaFree(bw.pc_pe);
      cudaFree(bw.pc_n);
      bw.pc_g = bw.pc_o = bw.pc_pe = nullptr;
      bw.pc_n = nullptr;
      bw.pc_cap = bw.pc_ncap = 0;
      if ((e = fpp::dev_malloc(&bw.pc_g, sizeof(uint32_t) * (size_t)npc)) != cudaSuccess ||
          (e = fpp::dev_malloc(&bw.pc_o, sizeof(uint32_t) * (size_t)npc)) != cudaSuccess ||
          (e = fpp::dev_malloc(&bw.pc_pe, sizeof(uint32_t) * (size_t)npc)) != cudaSuccess ||
          (e = fpp::dev_malloc(&bw.pc_n, sizeof(int) * (size_t)rq.nq)) != cudaSuccess)
        return fail(e, "alloc");
      bw.pc_cap = npc;
      bw.pc_ncap = rq.nq;
    }
    ProbeCutArgs pa;
    pa.ext_lv = bw.ext_lv;
    pa.ext_lb = bw.ext_lb;
    pa.ext_stride = ext_stride;
    pa.q_k = rq.q_k;
    pa.q_qprobes = rq.q_qprobes;
    pa.k_uniform = rq.k_uniform;
    pa.qprobes_uniform = rq.qprobes_uniform;
    pa.k_max = rq.k_max;
    pa.qprobes_max = rq.qprobes_max;
    pa.L = L;
    pa.bucket_off = di.bucket_off;
    pa.pc_g = bw.pc_g;
    pa.pc_o = bw.pc_o;
    pa.pc_pe = bw.pc_pe;
    pa.pc_n = bw.pc_n;
    pa.stride = rq.qprobes_max;
    if ((e = probe_cut_lists(pa, rq.nq, s)) != cudaSuccess) return fail(e, "probe cut launch");
  }
  BatchArgs a;
  a.Xc = di.Xc;
  a.ld = di.ld;
  if (rq.mode == kRowsF32) {
    a.Xrows = reinterpret_cast<const unsigned char*>(di.Xc);
    a.row_bytes = (size_t)di.ld * 4;
    a.nchunk = di.ld / 4;
  } else if (rq.mode == kRowsBF16) {
    a.Xrows = static_cast<const unsigned char*>(di.Xlp);
    a.row_bytes = (size_t)di.ld_lp * 2;
    a.nchunk = di.ld_lp / 8;
  } else {
    a.Xrows = static_cast<const unsigned char*>(di.Xlp);
    a.row_bytes = (size_t)di.ld_lp;
    a.nchunk = di.ld_lp / 16;
  }
  a.Xscale = di.Xlp_scale;
  a.flips = di.flips;
  a.bucket_off = di.bucket_off;
  a.ids = di.ids;
  a.n = P.n_points;
  a.d = d;
  a.L = L;
  a.D = D;
  a.log2D = log2D;
  a.NB = 4u * (uint32_t)D * (uint32_t)D;
  a.Q = rq.Q;
  a.nq = rq.nq;
  a.q_k = rq.q_k;
  a.q_qprobes = rq.q_qprobes;
  a.k_uniform = rq.k_uniform;
  a.qprobes_uniform = rq.qprobes_uniform;
  a.k_max = rq.k_max;
  a.qprobes_max = rq.qprobes_max;
  a.shortlist_mult = rq.shortlist_mult;
  a.out = rq.out;
  a.out_stride = rq.out_stride;
  a.out_v = rq.out_v;
  a.bitset = bw.bitset;
  a.nwords = bw.nwords;
  a.uniq = bw.uniq;
  a.score = bw.score;
  a.cap = bw.cap;
  a.gdump = bw.gdump;
  a.gheap_v = bw.gheap_v;
  a.gheap_i = bw.gheap_i;
  a.mmax = bw.mmax;
  a.work = bw.counters;
  a.status = bw.counters + 1;
  a.order = reorder ? bw.order : nullptr;
  a.tflips = (!big && rq.tc_rotation && rq.mode != kRowsF32 && F == 256) ? di.tflips : nullptr;
  a.glv = bw.glv;
  a.glb = bw.glb;
  a.list_cap = bw.list_cap;
  a.gprobe = bw.gprobe;
  a.gpo = bw.gpo;
  a.gpe = bw.gpe;
  a.probe_cap = bw.probe_cap;
  a.ggv = bw.ggv;
  a.ggc = bw.ggc;
  a.grhv = bw.grhv;
  a.grhi = bw.grhi;
  a.dump_probes = rq.dump_probes;
  a.dump_counts = rq.dump_counts;
  a.ext_lv = bw.ext_lv;
  a.ext_lb = bw.ext_lb;
  a.ext_stride = ext_stride;
  a.pc_g = pcut ? bw.pc_g : nullptr;
  a.pc_o = pcut ? bw.pc_o : nullptr;
  a.pc_pe = pcut ? bw.pc_pe : nullptr;
  a.pc_n = pcut ? bw.pc_n : nullptr;
  void* args[] = {&a};

  if (rq.stage_timing) {
    for (auto& ev : bw.tev)
      if (!ev && (e = cudaEventCreate(&ev)) != cudaSuccess) return fail(e, "event create");
    if (!split) {
      cudaEventRecord(bw.tev[0], s);
      cudaEventRecord(bw.tev[3], s);
    }
    cudaEventRecord(bw.tev[1], s);
  }
  const bool can_graph = rq.use_graph && !rq.dump_probes && !rq.dump_counts;
  BatchKey key{rq.Q, rq.nq, rq.q_k, rq.q_qprobes, rq.k_uniform, rq.qprobes_uniform, rq.k_max, rq.qprobes_max,
               rq.shortlist_mult, rq.out,
               rq.out_stride, rq.out_v, rq.mode, grid, kern, bw.bitset, a.order, a.tflips, s};
  // same launch shape (kernel, grid, stream, scratch): the captured graph is
  // replayed, with the kernel node's arguments updated when they changed
  const bool same_shape = bw.graph_exec && bw.key.kern == key.kern && bw.key.grid == key.grid &&
                          bw.key.stream == key.stream && bw.key.bitset == key.bitset;
  if (can_graph && same_shape) {
    if (!(bw.key == key)) {
      cudaKernelNodeParams kp = {};
      kp.func = const_cast<void*>(kern);
      kp.gridDim = dim3(grid);
      kp.blockDim = dim3(kBThreads);
      kp.sharedMemBytes = (unsigned)ks.smem;
      kp.kernelParams = args;
      if ((e = cudaGraphExecKernelNodeSetParams(bw.graph_exec, bw.graph_knode, &kp)) != cudaSuccess)
        return fail(e, "graph update");
      bw.key = key;
    }
    if ((e = cudaGraphLaunch(bw.graph_exec, s)) != cudaSuccess) return fail(e, "graph launch");
    res.graph_replayed = true;
  } else {
    if (can_graph) {
      if (bw.graph_exec) {
        cudaGraphExecDestroy(bw.graph_exec);
        bw.graph_exec = nullptr;
      }
      cudaGraph_t graph = nullptr;
      if ((e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return fail(e, "capture");
      cudaMemsetAsync(bw.counters, 0, sizeof(unsigned) * 2, s);
      cudaLaunchKernel(kern, dim3(grid), dim3(kBThreads), args, ks.smem, s);
      if ((e = cudaStreamEndCapture(s, &graph)) != cudaSuccess) return fail(e, "capture end");
      cudaGraphNode_t nodes[4];
      size_t nn = 4;
      bw.graph_knode = nullptr;
      if (cudaGraphGetNodes(graph, nodes, &nn) == cudaSuccess)
        for (size_t i = 0; i < nn; ++i) {
          cudaGraphNodeType t;
          if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) bw.graph_knode = nodes[i];
        }
      e = cudaGraphInstantiate(&bw.graph_exec, graph, 0);
      if (bw.graph) cudaGraphDestroy(bw.graph);
      bw.graph = graph;  // kept alive: the kernel node handle belongs to it
      if (e != cudaSuccess) return fail(e, "graph instantiate");
      if (!bw.graph_knode) {
        err.code = kErrCuda;
        err.msg = "batch query: captured graph has no kernel node";
        return err.code;
      }
      bw.key = key;
      if ((e = cudaGraphLaunch(bw.graph_exec, s)) != cudaSuccess) return fail(e, "graph launch");
    } else {
      if ((e = cudaMemsetAsync(bw.counters, 0, sizeof(unsigned) * 2, s)) != cudaSuccess) return fail(e, "memset");
      if ((e = cudaLaunchKernel(kern, dim3(grid), dim3(kBThreads), args, ks.smem, s)) != cudaSuccess)
        return fail(e, "launch");
    }
  }
  res.launches = (reorder ? 3 : 1) + (split ? 1 : 0) + (pcut ? 1 : 0);
  if (rq.stage_timing) {
    cudaEventRecord(bw.tev[2], s);
    if ((e = cudaEventSynchronize(bw.tev[2])) != cudaSuccess) return fail(e, "stage timing");
    cudaEventElapsedTime(&res.ms_hash, bw.tev[0], bw.tev[3]);
    cudaEventElapsedTime(&res.ms_prep, bw.tev[3], bw.tev[1]);
    cudaEventElapsedTime(&res.ms_fused, bw.tev[1], bw.tev[2]);
    if (vhash) {
      unsigned nx = 0;
      if ((e = cudaMemcpy(&nx, bw.counters + 2, sizeof(unsigned), cudaMemcpyDeviceToHost)) != cudaSuccess)
        return fail(e, "stage timing");
      res.tc_exact = nx;
    }
  }
  res.grid = grid;
  if (rq.check_status) {
    unsigned st[2] = {0, 0};
    if ((e = cudaMemcpyAsync(st, bw.counters, sizeof(st), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
      return fail(e, "status");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return fail(e, "batch kernel");
    res.overflow = (st[1] & 1u) != 0;
    res.bad_params = (st[1] & 2u) != 0;
  }
  return kOk;
}

}  // namespace fpp
