/*
 * voila_cuda.h -- C ABI of the CUDA flavor for VOILA's data-parallel hot path on one
 * NVIDIA B200 (sm_100a).
 *
 * Plain C: opaque handles, pointers and sizes only; no C++ or torch types cross it.  Every
 * call returns a status (VC_OK on success) and never throws; vc_last_error() returns the
 * calling thread's message for the last failed call.
 *
 * How the pieces map onto the reference (t1mm3/vldb_voila):
 *
 *   engine + tables   runtime::Database / Relation / Attribute with MinMaxInfo
 *                     (db-engine-paradigms/include/common/runtime/Database.hpp:28-75,
 *                      common/runtime/Types.hpp:11-33).  Columns live in HBM.
 *   plan text         the relalg tree (relalg.hpp:12-178) a benchmark query builds
 *                     (bench_tpch_rel.cpp), serialised as an S-expression
 *   query new/run/    the generated-library ABI voila_query_new/run/reset/free
 *   reset/free        (codegen.cpp:371-392; called by Compiler::_run, compiler.cpp:488-533)
 *   flavor string     the per-pipeline blend, computation_type=cuda(...) next to
 *                     scalar/avx512/vector(N) (blend_space_point.hpp:10-45)
 *   result text       QueryResult rows "a|b|c\n" (runtime_framework.cpp:77-111), compared
 *                     order-insensitively like Query::check_result (:220-280)
 *
 * Threading: one engine may be used from several host threads; calls on the same query
 * must be serialised by the caller.  Streams are passed as a plain cudaStream_t cast to
 * void* (NULL = the legacy default stream).
 */
#ifndef VOILA_CUDA_H
#define VOILA_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define VC_OK 0
#define VC_ERR_INVALID 1     /* bad argument, unknown table/column, malformed plan */
#define VC_ERR_CUDA 2        /* a CUDA runtime call failed (message names it) */
#define VC_ERR_CAPACITY 3    /* a device table ran out of slots */
#define VC_ERR_TIMEOUT 4     /* a bounded device wait gave up */
#define VC_ERR_COMPILE 5     /* NVRTC rejected generated code (log in the message) */
#define VC_ERR_UNSUPPORTED 6 /* valid plan the CUDA flavor does not handle (e.g. int64 overflow) */
#define VC_ERR_NO_DEVICE 7   /* no usable CUDA device */

/* column types (same values as vc_gen_spec.type) */
#define VC_U8 1
#define VC_I16 2
#define VC_I32 3
#define VC_I64 4
#define VC_STR 5 /* strings: 32-bit codes of the engine's string dictionary on the device */

typedef struct vc_engine vc_engine;
typedef struct vc_query vc_query;

/* Thread-local message of the last failing call ("" if none). Replaces the reference's
 * ASSERT/exception reporting (runtime.hpp:38-49, compiler.cpp:564-571). */
const char* vc_last_error(void);

/* Library version string. */
const char* vc_version(void);

/* ---------------------------------------------------------------- engine / database --- */

/* Creates an engine on CUDA device `device`.  Replaces constructing runtime::Database
 * (main.cpp:66) for the device side. */
int vc_engine_create(int device, vc_engine** out);
int vc_engine_destroy(vc_engine* eng);

/* Creates an engine without a device: vc_query_new then lowers the plan, generates the
 * kernels and compiles them for sm_100a (so code generation is testable on a build host),
 * but queries cannot run.  `sms` sizes grids as on a device with that many SMs. */
int vc_engine_create_offline(int sms, vc_engine** out);

/* Declares a table of `rows` rows (Relation with nrTuples, Database.hpp:66-75). */
int vc_table_create(vc_engine* eng, const char* table, int64_t rows);
int vc_table_drop(vc_engine* eng, const char* table);

/* Declares a column with its value domain [lo, hi] (Relation::insert + Attribute::minmax,
 * Database.hpp:32-44; read by the reference's codegen at codegen.cpp:11-19) and allocates
 * its device storage. */
int vc_column_add(vc_engine* eng, const char* table, const char* column, int type, int64_t lo, int64_t hi);

/* Uploads a string column (VC_STR): row r is bytes[offsets[r], offsets[r+1]) (rows + 1
 * offsets).  Strings are encoded into the engine's dictionary, shared by all its string
 * columns so equal strings of different tables get equal codes (joins and group keys on
 * strings compare codes); the column's domain becomes its codes' range.  Synchronous.
 * Replaces the reference's varchar attributes (runtime.hpp:150-224). */
int vc_column_upload_strings(vc_engine* eng, const char* table, const char* column, const char* bytes,
	const int64_t* offsets, int64_t rows);

/* Size of the engine's string dictionary, and the string of a code (string result columns
 * hold codes in vc_query_result_copy; vc_query_result_text prints the strings). */
int vc_dict_size(vc_engine* eng, int64_t* n);
int vc_dict_string(vc_engine* eng, int64_t code, char* buf, size_t cap, size_t* len);

/* A column's type, declared domain [lo, hi] and its table's row count (any pointer may be NULL). */
int vc_column_info(vc_engine* eng, const char* table, const char* column, int32_t* type, int64_t* lo, int64_t* hi,
	int64_t* rows);

/* Copies `rows` values from host memory into the column (Attribute::operator=,
 * Database.hpp:59-62).  Asynchronous on `stream`; pinned host memory gives full speed. */
int vc_column_upload(vc_engine* eng, const char* table, const char* column, const void* host, int64_t rows,
	void* stream);

/* Copies the column back to host memory (for checking). */
int vc_column_download(vc_engine* eng, const char* table, const char* column, void* host, int64_t rows,
	void* stream);

/* Uses caller-owned device memory (16-byte aligned, `rows` values) as the column; the
 * engine's own buffer is freed.  The memory must outlive every query that reads it. */
int vc_column_attach(vc_engine* eng, const char* table, const char* column, void* device_ptr);

/* Uses caller-owned pinned host memory (cudaHostAlloc / cudaHostRegister, 16-byte aligned,
 * `rows` values) as the column: queries created afterwards read it in place over PCIe, so a
 * step moves only the bytes its kernels touch (a probe chain gathers most columns only for
 * the rows that survive its first probes) instead of copying whole columns first.  The memory
 * must outlive every query that reads it; a later vc_column_attach makes the column
 * device-resident again for queries created after it.  No counterpart in the reference, whose
 * columns are host memory to begin with. */
int vc_column_attach_host(vc_engine* eng, const char* table, const char* column, const void* host_ptr);

/* Device address of the column's data. */
int vc_column_device_ptr(vc_engine* eng, const char* table, const char* column, void** out);

/* Fills the column on the device from a seeded generator (see vc_gen_spec in datagen.h:
 * kind, type, a, b, c, s, seed, n).  `zipf_cdf` (host, b doubles) is required for a skewed
 * VC_GEN_ZIPF column.  Stands in for the TPC-H/SSB import (Import.cpp:165-250). */
int vc_column_generate(vc_engine* eng, const char* table, const char* column, int32_t kind, int64_t a,
	int64_t b, int64_t c, double s, uint64_t seed, const double* zipf_cdf, void* stream);

/* Imports <dir>/<table>.tbl (pipe-separated text, one row per line: the TPC-H/SSB dbgen
 * format) as a new table: `schema` lists every field of a line in order as name:type (int,
 * bigint, date = YYYY-MM-DD as its Julian day number, decN = decimal as value * 10^N, char =
 * first byte) or "-" to skip it.  Parsed on `threads` host threads (0 = all) and cached as
 * raw column arrays <dir>/cached/<table>_<name>, which later imports read instead of the
 * text -- the reference's import path and cache layout (Import.cpp:165-250).  Each column's
 * declared domain is its observed [min, max] (the reference's MinMaxInfo).  *rows_out gets
 * the row count.  The upload is synchronous. */
int vc_table_import(vc_engine* eng, const char* table, const char* dir, const char* schema, int threads,
	int64_t* rows_out);

/* Host-side generator for the same columns: writes rows [begin, begin+count) into `out`
 * (element type `type`). */
int vc_gen_host(int32_t kind, int32_t type, int64_t a, int64_t b, int64_t c, double s, uint64_t seed, int64_t n,
	const double* zipf_cdf, int64_t begin, int64_t count, void* out);

/* Inverse-CDF table of Zipf(s) over n keys (n doubles). */
int vc_gen_zipf_cdf(double s, int64_t n, double* out);

/* Text description of a synthetic workload spec such as
 * "join_aggr:build=1500000,probe=6000000,sel=0.2,seed=2": tables, column generators with
 * their domains and the plan text.  Writes at most `cap` bytes; *len gets the full length. */
int vc_workload_describe(const char* spec, char* buf, size_t cap, size_t* len);

/* The base-table columns a plan scans, one "table column" line each, in the order the plan
 * names them: what a host uploads before vc_query_new (the reference binds the same
 * attributes when it sets up a generated query, runtime_struct.cpp:825-842). */
int vc_plan_columns(const char* plan, char* buf, size_t cap, size_t* len);

/* Spec strings of the seeded mixed batch (one per line). */
int vc_workload_batch(int count, uint64_t seed, int64_t min_rows, int64_t max_rows, char* buf, size_t cap,
	size_t* len);

/* ---------------------------------------------------------------- queries ------------- */

/* Translates plan text into fused CUDA pipelines with the flavor's knobs, generates and
 * compiles their kernels (NVRTC, cached by source) and allocates the query's device
 * state.  Replaces Compiler::_generate + call_cxx_compiler + voila_query_new
 * (compiler.cpp:19-57, :343-385; codegen.cpp:371-376).
 * flavor: "" or "cuda(key=value,...)" with keys threads, rows, load=ldg|tma, stages,
 * prefetch, compact, frows (survivors per thread in a compaction flush, 1..16),
 * aggr=auto|dense|global|cache|part|direct|dcache (part: partitioned group-by, histogram +
 * scatter + one shared-memory table per partition; direct: a group table indexed by the packed
 * key, no stored keys; dcache: the direct table behind the shared-memory cache), parts
 * (partitions of aggr=part, 16..2048), cache,
 * lowcard=combine|atomic|private|redux|regs|packed, pgroups (groups per CTA of lowcard=private|regs|packed),
 * build=auto|direct|staged|dense, hash=mix|voila, fill, dense, sinksmem, gcap (group table
 * slots), ocap (result rows of an emitting plan), probe (1..32 lanes that probe one join key
 * together), grid, minctas (CTAs per SM the main kernel's registers must allow),
 * stream=ldg|noalloc (column loads through the read-only path, or without L1 allocation so that
 * probed tables keep L1), graph.
 * VC_ERR_INVALID for an unknown or out-of-range knob; VC_ERR_UNSUPPORTED when the flavor's
 * shared memory exceeds the device's per-CTA limit or build=dense meets a large key space. */
int vc_query_new(vc_engine* eng, const char* plan, const char* flavor, vc_query** out);

/* Launches the query's pipelines on `stream` (voila_query_run, codegen.cpp:390; the
 * pipelines run in order like Query::run, runtime_framework.cpp:166-198).  Asynchronous:
 * results are read with vc_query_result_*. */
int vc_query_run(vc_query* q, void* stream);

/* Clears the query's state between runs (voila_query_reset, codegen.cpp:391).  vc_query_run
 * resets the device state itself, so this only drops the host copy of the last result. */
int vc_query_reset(vc_query* q);

/* voila_query_free (codegen.cpp:392). */
int vc_query_free(vc_query* q);

/* Waits for the last run and reports its result shape (rows x cols, int64 values). */
int vc_query_result_shape(vc_query* q, int64_t* rows, int32_t* cols);

/* Copies the last result, column-major (cols x rows int64), into `out` (capacity `cap`
 * values). */
int vc_query_result_copy(vc_query* q, int64_t* out, int64_t cap);

/* The last result as QueryResult text (runtime_framework.cpp:77-111): decimal values
 * separated by '|', one row per line, in device order (compare after sorting lines). */
int vc_query_result_text(vc_query* q, char* buf, size_t cap, size_t* len);

/* JSON description: pipelines, kernels, flavor, algorithmic bytes, generated source size. */
int vc_query_info(vc_query* q, char* buf, size_t cap, size_t* len);

/* Lowers plan text with a flavor (no code generation, no compilation) and describes its
 * pipelines as JSON: table, rows, columns, filters, probes (joinN among them), rows of the
 * probed builds, sink kind, aggregates, key domain, groups bound, scanned bytes.  The
 * features the flavor chooser works from. */
int vc_plan_describe(vc_engine* eng, const char* plan, const char* flavor, char* buf, size_t cap, size_t* len);

/* Generated CUDA source of the query (for inspection and tests). */
int vc_query_source(vc_query* q, char* buf, size_t cap, size_t* len);

/* Per-launch device times of the last run, in launch order (enable first with
 * vc_query_profile).  `names` receives kernel names separated by '\n'. */
int vc_query_profile(vc_query* q, int enable);

/* Runs the query `reps` times on `stream` and stores each run's device time (CUDA events
 * around the run) in ms_out[0..reps); with flush_l2 a 256 MiB buffer is written before every
 * run so inputs come from HBM.  The timing primitive of the autotuner (the reference's
 * timed hot repetitions, compiler.cpp:521-575). */
int vc_query_time(vc_query* q, int reps, int flush_l2, void* stream, float* ms_out, int cap);

/* Reads `bytes` of device memory once, as fast as a plain streaming read can (16-byte loads,
 * several in flight per thread, whole waves of CTAs), and XORs the words into *device_out.
 * The bandwidth floor a pipeline over the same bytes is measured against; no counterpart in
 * the reference (its CPU baseline has no device roofline).  Asynchronous on `stream`. */
int vc_stream_read(const void* device_buf, int64_t bytes, unsigned long long* device_out, void* stream);

/* ---------------------------------------------------------------- no allocation ------- */

/* The hash join + global aggregate pipeline (a join_aggr query: build rows with
 * build_attr < attr_threshold form a Join01 table on build_key; every probe row whose
 * probe_key is in it contributes probe_val) without any device allocation.  This entry point
 * has no counterpart in the reference.  It is for callers that cannot call cudaMalloc --
 * code running where allocation is forbidden or unsafe (host callbacks, allocator-owned
 * device memory, allocation-free service paths).  All pointers are caller-owned device
 * memory; out receives 3 int64: sum(probe_val) over matches, the match count, and error
 * bits (0 = none).  The error bits are the only report of a table that ran out of probes:
 * a VC_OK return means the launch succeeded, so callers must check out[2] == 0 (after the
 * stream has finished) before using out[0] and out[1].
 * Limit: at most 2,097,152 build rows (the join table is a static 4 Mi-slot, 32 MiB device
 * array that every GPU loading the library keeps until the process exits); larger inputs fail
 * with VC_ERR_INVALID.  The first call on a device looks the arrays' addresses up
 * (cudaGetSymbolAddress) and should come before any stream capture.  All calls on a device
 * share the arrays and the last call's contents remain (each call clears what it uses);
 * calls that overlap on the GPU race and give wrong results. */
int vc_join_aggr_noalloc(const int32_t* build_key, const int32_t* build_attr, int64_t build_rows,
	int32_t attr_threshold, const int32_t* probe_key, const int64_t* probe_val, int64_t probe_rows, int64_t* out,
	void* stream);

/* ---------------------------------------------------------------- batches ------------- */

/* Many queries in one persistent kernel driven by a device work queue, launched from a
 * captured CUDA graph.  The reference runs queries one at a time, each pipeline fanned out
 * over threads (runtime_framework.cpp:166-198); a batch instead fuses every pipeline of every
 * query (each with its own flavor; threads per CTA shared) into one launch whose CTAs pull
 * tile ranges in dependency order (join builds before their probes, group tables before
 * their extraction).  The queries keep their device state and results: after
 * vc_batch_run + vc_batch_wait, vc_query_result_* read each query's rows.  The queries must
 * outlive the batch.  flavors may be NULL (each query's own) or hold one flavor per query
 * (NULL entries = the query's own).  tiles_per_item: tiles of a pipeline per work item.
 * Inside a batch, loads are plain (load=ldg), lowcard=private|regs|packed run as lowcard=combine and
 * cache= is capped at 256 slots, since every CTA reserves the largest shape's shared memory;
 * a partitioned group-by (aggr=part) runs through a global group table, allocated on first
 * use. */
typedef struct vc_batch vc_batch;
int vc_batch_new(vc_query** queries, int n, const char** flavors, int threads, int64_t tiles_per_item, vc_batch** out);
/* vc_batch_new whose queries with a pipeline of at least solo_rows rows (0 = none) run as
 * their own launches, with their own flavors' kernels, on the same stream right after the
 * persistent kernel that runs the rest: a pipeline that fills the GPU by itself gains nothing
 * from the batch's lean shared shapes (a solo query runs the flavor it was created with; its
 * entry in flavors is not used).  vc_batch_info reports "batched" and "solo" counts;
 * vc_batch_latencies gives a solo query the time from the batch's start to its end.  No
 * counterpart in the reference, which runs queries one at a time. */
int vc_batch_new_split(vc_query** queries, int n, const char** flavors, int threads, int64_t tiles_per_item,
	int64_t solo_rows, vc_batch** out);
int vc_batch_run(vc_batch* b, void* stream);
/* Waits for the run; VC_ERR_TIMEOUT if a bounded dependency wait gave up. */
int vc_batch_wait(vc_batch* b);
/* Completion time of each query, in microseconds since the batch kernel started. */
int vc_batch_latencies(vc_batch* b, double* us, int n);
int vc_batch_info(vc_batch* b, char* buf, size_t cap, size_t* len);
/* The generated CUDA source of the batch's persistent kernel. */
int vc_batch_source(vc_batch* b, char* buf, size_t cap, size_t* len);
/* The work queue in claim order, 8 int64 per item: shape (-1 = clear), done-counter waited
 * for (-1 = none), its target, done-counter incremented, items of the stage, tile (or byte)
 * range begin and end, parameter offset.  *n = item count; out may be NULL. */
int vc_batch_items(vc_batch* b, int64_t* out, int64_t cap, int64_t* n);
/* Longest time (ns, 1 us .. 60 s; default 2 s) that a work item waits for its dependency
 * before the batch gives up on it: the item is skipped, the batch's error word records the
 * timeout and vc_batch_wait returns VC_ERR_TIMEOUT.  Replaces the reference's fork-isolated
 * timeout classification (safe_env.cpp:66-187) for the device side. */
int vc_batch_set_wait_limit(vc_batch* b, uint64_t ns);
/* Test hook for the timeout path, made on the host: with hold != 0, work item `index` (claim
 * order, as vc_batch_items lists it) waits for a dependency that never completes, so its
 * bounded wait runs out on the next run; hold == 0 restores it.  No counterpart in the
 * reference. */
int vc_batch_hold_item(vc_batch* b, int64_t index, int hold);
int vc_batch_free(vc_batch* b);

/* ---------------------------------------------------------------- flavor chooser ------ */

/* A small multi-layer perceptron (in -> hidden -> hidden -> out, ReLU), trained and run on
 * the GPU by the library's own kernels.  It maps a pipeline's features to the predicted
 * relative time of every candidate flavor; the caller picks the argmin.  It stands beside
 * the exhaustive search over blends that the reference's explorer performs
 * (explorer.cpp:111-134, :352-426), which remains the fallback and the yardstick of its choices. */
typedef struct vc_mlp vc_mlp;

/* Glorot-uniform weights from `seed`, zero biases. */
int vc_mlp_create(int device, int n_in, int n_hidden, int n_out, uint64_t seed, vc_mlp** out);
int vc_mlp_free(vc_mlp* m);
int vc_mlp_num_params(vc_mlp* m, int64_t* n);
/* Parameters flattened as W1[in][hidden], b1, W2[hidden][hidden], b2, W3[hidden][out], b3. */
int vc_mlp_get_params(vc_mlp* m, float* out, int64_t cap);
int vc_mlp_set_params(vc_mlp* m, const float* in, int64_t n);
/* Masked mean squared error of (X[n][in] -> targets T[n][out]) and its gradient with respect
 * to every parameter (same layout as the parameters).  mask may be NULL (all ones). */
int vc_mlp_loss_grad(vc_mlp* m, const float* X, const float* T, const float* mask, int n, float* loss, float* grads);
/* Adam training, shuffled mini-batches; *final_loss = loss over all n samples after training. */
int vc_mlp_train(vc_mlp* m, const float* X, const float* T, const float* mask, int n, int epochs, int batch, float lr,
	uint64_t seed, float* final_loss);
int vc_mlp_predict(vc_mlp* m, const float* X, int n, float* Y);
int vc_query_timings(vc_query* q, float* ms, int cap, int* n, char* names, size_t names_cap);

#ifdef __cplusplus
}
#endif

#endif
