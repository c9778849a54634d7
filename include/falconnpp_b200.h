/* falconnpp_b200.h — C ABI of the B200 Falconn++ index (one GPU).
 *
 * Every entry point is plain C: opaque handle, plain pointers and sizes, and
 * an int status (0 = success, negative = error; fpp_last_error() then returns
 * a message for the calling thread).  Matrices use the reference's layout:
 * a d x n column-major float32 matrix, i.e. n points of d contiguous floats.
 *
 * Each function names the reference interface it replaces (paths relative to
 * the reference project root).  Calls on one handle are serialised.
 */
#ifndef FALCONNPP_B200_H
#define FALCONNPP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fpp_index fpp_index;

enum {
  FPP_OK = 0,
  FPP_ERR_INVALID_ARGUMENT = -1,
  FPP_ERR_NOT_BUILT = -2,
  FPP_ERR_CUDA = -3,
  FPP_ERR_OUT_OF_MEMORY = -4,
  FPP_ERR_UNSUPPORTED = -5,
  FPP_ERR_NON_FINITE = -6,
  FPP_ERR_DEVICE = -7
};

/* Replaces FalconnPP::FalconnPP(int n, int d), src/FalconnPP.h:80-83
 * (python: FalconnPP(n_points, n_features), python/python_wrapper.cpp:16).
 * Binds the handle to the current CUDA device. */
int fpp_create(int n_points, int n_features, fpp_index** out);

/* Replaces FalconnPP::~FalconnPP, src/FalconnPP.h:131.  Frees all device memory. */
void fpp_destroy(fpp_index* h);

/* Replaces FalconnPP::Index2Layers, src/FalconnPP.h:85-100
 * (python: setIndexParam(n_tables, n_proj, bucket_minSize, bucket_scale, iProbes,
 * n_threads=8, random_seed=-1), python/python_wrapper.cpp:19-22).
 * random_seed = -1 seeds from the wall clock exactly like the reference.
 * Rejects what the reference leaves undefined: n_proj not a power of two,
 * fhtDim > 1024, iProbes outside [1, min(32, n_proj)]. */
int fpp_set_index_param(fpp_index* h, int n_tables, int n_proj, int bucket_minSize, float bucket_scale,
                        int iProbes, int n_threads, int random_seed);

/* Replaces FalconnPP::set_qProbes, src/FalconnPP.h:113-115. */
int fpp_set_qprobes(fpp_index* h, int qProbes);

/* Replaces FalconnPP::set_threads, src/FalconnPP.h:117-123.  Stored and
 * reported; the GPU path does not use host threads. */
int fpp_set_threads(fpp_index* h, int n_threads);

/* Replaces FalconnPP::clear, src/FalconnPP.h:102-111. */
int fpp_clear(fpp_index* h);

/* Replaces FalconnPP::build2Layers_1D, src/FalconnPP.cpp:21-303
 * (python: build(dataset), python/python_wrapper.cpp:28).
 * dataset: host memory, d x n column-major float32 (n points of d floats). */
int fpp_build(fpp_index* h, const float* dataset);

/* Same as fpp_build with the dataset already in device memory; stream may be
 * NULL (the handle's own stream).  Returns after the index is complete. */
int fpp_build_device(fpp_index* h, const float* d_dataset, void* stream);

/* Replaces FalconnPP::query2Layers_1D, src/FalconnPP.cpp:310-707
 * (python: query(queries, n_neighbors, verbose=False), python/python_wrapper.cpp:29-30).
 * queries: host, d x n_queries column-major; out: host, n_queries x n_neighbors
 * int32 row-major, each row in descending inner product, 0-padded.
 * verbose = 1 prints the reference's statistics and writes its
 * 1D_Top_<k>_D_..._qProbe_<q>.txt file to the working directory
 * (FalconnPP.cpp:682-703). */
int fpp_query(fpp_index* h, const float* queries, int n_queries, int n_neighbors, int verbose, int32_t* out);

/* Same as fpp_query with queries and out in device memory; asynchronous with
 * respect to the host only as far as the kernels allow (the call returns once
 * the results are written).  stream may be NULL. */
int fpp_query_device(fpp_index* h, const float* d_queries, int n_queries, int n_neighbors, int32_t* d_out,
                     void* stream);

/* Message of the last failing call on this thread ("" if none). */
const char* fpp_last_error(void);

/* Index facts: out[0] fhtDim, out[1] stored ids, out[2] largest stored bucket,
 * out[3] buckets (n_tables * 4 * n_proj^2), out[4] built (0/1), out[5] device,
 * out[6] n_tables, out[7] n_proj, out[8] iProbes (the first n are written). */
int fpp_get_info(fpp_index* h, long long* out, int n);

/* Statistics of the last build (kind 0) or query (kind 1) as doubles.
 * build: ms_center, ms_hash, ms_sort, ms_csr, ms_total, repaired buckets,
 *        limited buckets (FalconnPP.cpp:241), points per table / n (:296);
 * query: candidates, unique candidates, empty probed buckets, probes,
 *        probe-cut replays, top-k replays (all summed over the queries),
 *        kernels launched, then (with the "stage_timing" option) the CUDA-event
 *        milliseconds of the hashing, probe-selection and gather/rerank kernels
 *        (batched form: the hash kernel, the order and probe-cut kernels, and
 *        the fused kernel), and (batched form with stage timing) the tables
 *        the verified tensor-core hash re-hashed in FP32, summed over the
 *        queries. */
int fpp_get_stats(fpp_index* h, int kind, double* out, int n);

/* Tuning and test switches: "exact_bucket_order" (default 1: bucket contents
 * in the reference's heap order even among equal scores; 0: ascending id among
 * equal scores, the kept set is identical either way), "tables_per_chunk",
 * "stage_timing" (0/1: CUDA events around each query kernel), "use_graph"
 * (0/1: batched form captured into a CUDA graph and replayed for repeated
 * shapes; the stream must not be the legacy default stream), "blocks_per_sm"
 * (batched form: resident blocks per SM, 0 = occupancy limit),
 * "reorder_queries" (default 1: the batched form processes a batch grouped by
 * the first table's first-layer bucket code, so queries in flight together
 * share buckets and rows in L2; results are unchanged), "split_hash" (default
 * 1: the batched form hashes in its own exact FP32 kernel, then runs the probe
 * cut of every query in its own kernel, before the fused gather / rerank /
 * top-k kernel; 0: one fused kernel that also rotates and hashes; the results
 * are the same), "tc_hash" (default
 * 1: with the split hash, fhtDim 256, n_tables <= 128 and 2 qProbes <=
 * n_tables, the hash kernel rotates on the tensor cores with FP16 operands,
 * bounds the error of every table's score from the query's norm, and hashes
 * again in the reference's FP32 arithmetic every table whose score can reach
 * the probe cut (every table when exact scores tie at the cut); the probes
 * and their scores are those of the exact hash; 0: the exact FP32 hash of
 * every table), "tc_rotation"
 * (default 0, opt-in: the batched BF16/FP8 form with fhtDim 256 and one probe
 * per table rotates on the tensor cores with FP16 operands and FP32
 * accumulation instead of the reference's FP32 arithmetic; its probes can then
 * differ from the reference's where two rotated coordinates or two bucket
 * scores are within about 1e-3 of each other.  With the default, every form
 * hashes in exact FP32 and probes the reference's buckets),
 * "inject_alloc_failure" (test switch, process-wide: n >= 1 makes the n-th
 * device allocation from now on fail once with FPP_ERR_OUT_OF_MEMORY, on the
 * host and without touching the GPU; 0 disarms). */
int fpp_set_option(fpp_index* h, const char* key, long long value);

/* Prints the build report the reference writes to stdout after
 * build2Layers_1D (src/FalconnPP.cpp:23-30, :275-301) for the last build. */
void fpp_print_build_report(fpp_index* h);

/* Parity dumps (host buffers).
 * fpp_dump_bits: bitHD1/bitHD2 (src/FalconnPP.h:61-68), n_tables*3*fhtDim bytes each.
 * fpp_dump_center: the d floats subtracted from the data (FalconnPP.cpp:33).
 * fpp_dump_tables: bucket_start[n_buckets+1] (CSR offsets, bucket size =
 *   difference, equal to the reference's uint16 bucket size) and ids[stored ids]. */
int fpp_dump_bits(fpp_index* h, uint8_t* bitHD1, uint8_t* bitHD2);
int fpp_dump_center(fpp_index* h, float* center);
int fpp_dump_tables(fpp_index* h, uint32_t* bucket_start, int32_t* ids);

/* fpp_build with the per-(table, point) hash codes captured: codes/scores are
 * [n_tables][n_points][iProbes] in the drain order of the reference's minQue
 * (FalconnPP.cpp:196-201). */
int fpp_build_dump_hash(fpp_index* h, const float* dataset, int32_t* codes, float* scores);

/* fpp_query with intermediate results captured (any pointer may be NULL):
 * topk_val [nq][k] scores; probes / probe_val [nq][qProbes] probed global
 * bucket ids (the probed set; its order is the pop order only where scores
 * differ); stats [nq][4] = candidates, unique candidates, empty buckets,
 * probes; cands [nq][cand_cap] the unique candidate ids (unordered, -1 padded).
 * cand_cap must be at least the largest unique-candidate count of the batch. */
int fpp_query_dump(fpp_index* h, const float* queries, int n_queries, int n_neighbors, int32_t* out,
                   float* topk_val, uint32_t* probes, float* probe_val, long long* stats, int32_t* cands,
                   long long cand_cap);

/* Selects the implementation behind fpp_query / fpp_query_device (and the
 * Python query()).  form 0 (default): the plain FP32 path of three kernels,
 * bit-exact with src/FalconnPP.cpp:310-707.  form 1: the batched path, one
 * persistent fused kernel per batch (rotate, hash, probe, gather, rerank,
 * top-k) with dynamic scheduling; precision 0 reranks in FP32 and equals the
 * plain path bit for bit; precision 1 (BF16) and 2 (FP8-E4M3 with a per-row
 * scale) rerank the candidates in low precision with FP32 accumulation and
 * re-score the best shortlist_mult * k of them in exact FP32.  Every form
 * gets the probes of the reference's FP32 hash (the batched form's
 * tensor-core rotation under "tc_hash" re-hashes in FP32 every table that can
 * reach the probe cut; only the opt-in "tc_rotation" option departs from
 * it), so every form probes the same buckets and gathers the same
 * candidates; only the low-precision rerank differs.
 * Extends query2Layers_1D; no reference counterpart for the batched form. */
int fpp_set_query_form(fpp_index* h, int form, int precision, int shortlist_mult);

/* Batched form with per-query k and qProbes (mixed batches).  d_k and
 * d_qprobes are device int32 arrays of n_queries entries (NULL: every query
 * uses k_max / qprobes_max); k_max and qprobes_max bound them.  d_out is
 * n_queries x out_stride int32 (first k of each row written, descending
 * score, 0-padded), d_out_val the matching scores or NULL.  Uses the handle's
 * precision and shortlist setting.  Returns after the results are written.
 * Limits: ceil(sqrt(ceil(2 qProbes / n_tables))) <= min(32, n_proj),
 * n_tables <= 512, k * shortlist_mult <= 1024.  Batches with qProbes > 1024,
 * n_tables * ceil(2 qProbes / n_tables) > 1024 or more than 16 probes per
 * layer run the big-list instances, whose lists live in global scratch. */
int fpp_query_batched(fpp_index* h, const float* d_queries, int n_queries, const int32_t* d_k,
                      const int32_t* d_qprobes, int k_max, int qprobes_max, int32_t* d_out, int out_stride,
                      float* d_out_val, void* stream);

/* Parity dump of the batched form (no reference counterpart): runs the
 * handle's batched configuration (precision, shortlist, the handle's qProbes,
 * uniform k) on device queries and also writes, per query, the probed global
 * bucket ids (d_probes, n_queries x qProbes, the probed set in no particular
 * order) and d_counts (n_queries x 2: candidates, unique candidates).  These
 * equal fpp_query_dump's probes and counts (src/FalconnPP.cpp:540-606) in
 * every precision: only the rerank differs between the forms.  d_out_val,
 * d_probes and d_counts may be NULL.  No graph is used.  Returns after the
 * results are written. */
int fpp_query_batched_dump(fpp_index* h, const float* d_queries, int n_queries, int n_neighbors, int32_t* d_out,
                           float* d_out_val, uint32_t* d_probes, uint32_t* d_counts, void* stream);

/* Autotuner of the batched form (no reference counterpart).  On a sample of
 * device queries it times the batched form over precision {BF16, FP8} x
 * shortlist multiple {2,4} x resident fused blocks per SM {1,2,3} (each
 * block works on one query at a time, so this is the queries in flight per
 * SM) x exact hash in its own kernel or inside the fused one x query grouping
 * on/off, against the FP32 exact batched result, and keeps the fastest
 * configuration whose top-k ids agree with the exact ones on at least
 * min_agreement of the ids (the FP32 configuration itself when none does).
 * The hash and grouping choices change no result; precision and shortlist
 * can.  The handle is switched to the batched form with that configuration.
 * report (may be NULL): double[8] = best ms for the sample, blocks per SM
 * (0 = occupancy limit), precision, shortlist multiple, agreement,
 * configurations tried, split hash (0/1), query grouping (0/1). */
int fpp_autotune(fpp_index* h, const float* d_queries, int n_queries, int k, double min_agreement, double* report,
                 void* stream);

/* Serving loop with continuous batching (no reference counterpart).
 * A worker thread packs submitted requests (1..max_batch queries each, their
 * own k <= k_max and qProbes <= qprobes_max) into mixed batches of the
 * batched form and launches them on n_streams concurrent streams; requests
 * that arrive while batches run are admitted as stream slots free up, as
 * long as the queries and results in flight stay within
 * memory_budget_bytes (a request is always admitted into an empty slot).
 * Uses the handle's precision and shortlist setting at creation; do not
 * rebuild or clear the index while a server exists.  Creation runs one
 * batch of max_batch zero queries per stream, which sizes each stream's
 * workspace for the largest batch, so serving allocates nothing.  queries / out are host
 * buffers that must stay valid until fpp_server_wait returns for the ticket;
 * wait on each ticket exactly once.  latency_ms: submit to results written. */
typedef struct fpp_server fpp_server;
int fpp_server_create(fpp_index* h, int n_streams, long long memory_budget_bytes, int max_batch, int k_max,
                      int qprobes_max, fpp_server** out);
int fpp_server_submit(fpp_server* s, const float* queries, int n_queries, int k, int qprobes, int32_t* out,
                      long long* ticket);
int fpp_server_wait(fpp_server* s, long long ticket, double* latency_ms);
/* out[0] launches, out[1] queries, out[2] requests submitted, out[3] requests waiting. */
int fpp_server_stats(fpp_server* s, double* out, int n);
void fpp_server_destroy(fpp_server* s);

/* Exact maximum-inner-product top-k in FP64 on the GPU: the ground truth of
 * recall measurements.  Replaces BF::mips_topK, src/BF.cpp:17-86 (which is
 * FP32 on the CPU); ties are broken by ascending id.  d_X: n_points x
 * n_features float32 (the raw or the centred data: the ranking is the same),
 * d_Q: n_queries x n_features, d_out: n_queries x k int32 ids, d_out_val
 * (may be NULL): the FP64 inner products.  Independent of any index handle.
 * Limits: k <= 256, n_features <= 1024.  Returns after the results are
 * written. */
int fpp_bruteforce_topk_f64(const float* d_X, long long n_points, int n_features, const float* d_Q, int n_queries,
                            int k, int32_t* d_out, double* d_out_val, void* stream);

/* Brute-force block rerank in low precision on the tensor cores (no
 * reference counterpart; the exact model is BF::mips_topK, src/BF.cpp:17-86).
 * Scores every indexed point against every query with tcgen05 MMAs over the
 * index's centred rows in BF16 (precision 1) or FP8-E4M3 with per-row and
 * per-query FP32 scales (precision 2), FP32 accumulation, keeps the best
 * k * shortlist_mult per query, re-scores them in exact FP32 (the query
 * path's dot order) and returns the top k by (score desc, id asc): d_out
 * n_queries x k int32, d_out_val (may be NULL) the FP32 scores.  d_queries:
 * n_queries x n_features device floats.  Limits: k * shortlist_mult <= 256,
 * n_features <= 256 (BF16) / 512 (FP8).  Returns after the results are
 * written. */
int fpp_bruteforce_topk_lowp(fpp_index* h, const float* d_queries, int n_queries, int n_neighbors, int precision,
                             int shortlist_mult, int32_t* d_out, float* d_out_val, void* stream);

/* Index persistence (no counterpart in the reference, which rebuilds its
 * index on every run): fpp_save writes a built index (parameters, sign bits,
 * centre, centred rows, CSR bucket offsets and ids) to one binary file;
 * fpp_load reads it into a handle created for the same n_points x
 * n_features, which is then built (setIndexParam is not needed).  fpp_load
 * checks the header, the file size, the sign bits, the offsets (from 0,
 * non-decreasing, ending at the id count) and every id (in [0, n_points))
 * before the handle uses them; a rejected file leaves the handle's previous
 * index untouched if the header or sign bits fail, and the handle unbuilt if
 * a later section fails.  Query results after a load equal those of the
 * index that was saved. */
int fpp_save(fpp_index* h, const char* path);
int fpp_load(fpp_index* h, const char* path);

/* The reference's text matrix formats (src/Utilities.cpp:13-61), for the
 * command-line workflow.  fpp_load_txt reads n_points lines of n_features
 * whitespace-separated floats into out (n_points x n_features, one point per
 * row: the d x n column-major matrix of loadtxtData); like the reference it
 * leaves 0 where the file runs short, and *n_read (may be NULL) reports how
 * many values it read; a missing file is an error (the reference exits).
 * fpp_output_file writes topk (n_queries x k int32) one query per line, each
 * id followed by a space, as outputFile does for the K x Q matrix the
 * reference's query returns. */
int fpp_load_txt(const char* path, int n_points, int n_features, float* out, long long* n_read);
int fpp_output_file(const char* path, const int32_t* topk, int n_queries, int k);

/* No counterpart in the reference.  The gather, deduplicate, rerank and top-k
 * stage of fpp_query for callers that cannot allocate device memory: a
 * serving thread that must not stall on cudaMalloc / cudaFree (they
 * synchronise the device), or a host process whose device memory belongs to
 * another allocator.  It allocates nothing: its scratch is a 64 MiB
 * __device__ array that every GPU loading the library holds until exit.
 * d_queries: n_queries x n_features floats; d_probes: n_queries x n_probes
 * global bucket ids (the probes fpp_query_dump reports); d_out: n_queries x
 * n_neighbors int32, the same top-k fpp_query gives for those probes.  All
 * three in device memory.  The first call on a device looks up the scratch
 * address.  The call waits for its kernel before it returns.  Calls whose
 * kernels overlap on one GPU race on the shared scratch.  Rejects
 * n_neighbors > 1024, n_features > 1024, n_points beyond the scratch (about
 * 500M), probe ids outside [0, n_tables * 4 * n_proj^2) (read as empty
 * buckets, FPP_ERR_INVALID_ARGUMENT), and queries with more unique
 * candidates than a block's share (65536 when n_points allows; the row is
 * zeroed and FPP_ERR_UNSUPPORTED returned). */
int fpp_rerank_probes_noalloc(fpp_index* h, const float* d_queries, int n_queries, const uint32_t* d_probes,
                              int n_probes, int n_neighbors, int32_t* d_out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FALCONNPP_B200_H */
