/*
 * Host-side internals of the CUDA flavor: the relational plan mirror, the lowered
 * pipelines, the kernel generator's output and the runtime objects behind the C ABI.
 */
#ifndef VOILA_B200_ENGINE_INTERNAL_HPP
#define VOILA_B200_ENGINE_INTERNAL_HPP

#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "datagen.h"
#include "sexpr.hpp"

namespace vc {

/* An error that maps to a C ABI status code. */
struct Error : std::runtime_error {
	int code;
	Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define VC_CHECK_CUDA(call)                                                                       \
	do {                                                                                          \
		cudaError_t _e = (call);                                                                  \
		if (_e != cudaSuccess) {                                                                  \
			throw ::vc::Error(2 /* VC_ERR_CUDA */, std::string(#call) + ": " + cudaGetErrorString(_e)); \
		}                                                                                         \
	} while (0)

/* ------------------------------------------------------------------ relational plan ---- */

/* Mirror of the reference's relalg expressions (relalg.hpp:12-74). */
struct RelExpr {
	enum Kind { Const, ColId, Fun, Assign } kind;
	std::string text;                         /* constant literal, column id, function or assign name */
	std::vector<std::shared_ptr<RelExpr>> args;
};
using RelExprP = std::shared_ptr<RelExpr>;

/* Mirror of the reference's relalg operators (relalg.hpp:76-172). */
struct RelOp {
	enum Kind { Scan, Select, Project, HashAggr, HashJoin } kind;
	std::string table;                        /* Scan */
	std::vector<std::string> columns;         /* Scan */
	RelExprP predicate;                       /* Select */
	std::vector<RelExprP> exprs;              /* Project: projections; HashAggr: keys */
	std::vector<RelExprP> aggregates;         /* HashAggr */
	bool global = false;                      /* HashAggr::Global */
	bool join01 = true;                       /* HashJoin::Join01 (else JoinN) */
	std::vector<RelExprP> left_keys, left_payl, right_keys, right_payl;
	std::shared_ptr<RelOp> left, right;       /* child / probe side, build side */
};
using RelOpP = std::shared_ptr<RelOp>;

RelOpP parse_plan(const std::string& text);

/* ------------------------------------------------------------------ database ----------- */

struct Column {
	std::string name;
	int type = VC_TYPE_I32;
	int64_t lo = 0, hi = 0;   /* declared domain (the reference's MinMaxInfo); strings: their codes */
	void* dev = nullptr;      /* device data */
	bool owned = false;
	bool str = false;         /* holds string dictionary codes (VC_STR, or a key of one carried on) */
	bool host = false;        /* pinned host memory the kernels read in place over PCIe */
};

struct Table {
	std::string name;
	int64_t rows = 0;
	std::vector<Column> cols;
	Column* find(const std::string& c) {
		for (auto& x : cols) {
			if (x.name == c) {
				return &x;
			}
		}
		return nullptr;
	}
};

/* Engine-wide string dictionary: every string column of an engine is stored on the device as
 * 32-bit codes of one dictionary, so string equality, joins and group keys compare codes and
 * results are decoded on the host. */
struct StringDict {
	std::vector<std::string> strings;
	std::unordered_map<std::string, int32_t> codes;
	int32_t encode(const std::string& s) {
		auto it = codes.find(s);
		if (it != codes.end()) {
			return it->second;
		}
		if (strings.size() >= (size_t)INT32_MAX) {
			throw std::runtime_error("string dictionary is full");
		}
		const int32_t c = (int32_t)strings.size();
		strings.push_back(s);
		codes.emplace(s, c);
		return c;
	}
	int32_t find(const std::string& s) const {
		auto it = codes.find(s);
		return it == codes.end() ? -1 : it->second;
	}
};

/* ------------------------------------------------------------------ lowered pipelines -- */

struct Bounds {
	__int128 lo = 0, hi = 0;
};

struct BExpr;
using BExprP = std::shared_ptr<BExpr>;

struct BExpr {
	enum Kind { Col, Const, ProbeOut, Fun } kind;
	int col = -1;              /* Col: index into Pipeline::cols */
	int64_t cval = 0;          /* Const */
	int probe = -1, pidx = -1; /* ProbeOut: op index, payload index */
	std::string fn;            /* Fun: lt le gt ge eq ne and or add sub mul; inset; shr lowbits extract_year */
	std::vector<BExprP> args;
	Bounds b;
	bool boolean = false;
	bool str = false;          /* a string: a dictionary code (Col, ProbeOut) or a string constant */
	std::string sval;          /* string constant */
	int aux = -1;              /* inset: index of the code bitmap in LoweredPlan::bitmaps */
};

struct JoinDesc {
	int id = 0;
	std::string build_table;
	int64_t build_rows = 0;          /* upper bound of inserted rows */
	std::vector<Bounds> key_b, pay_b;
	std::vector<int> key_shift, pay_shift;
	int key_bits = 0, pay_bits = 0;
	bool key64 = false, pay64 = false;
	bool join01 = true;
	/* device state */
	void* table = nullptr;           /* JoinSlot array, capacity for build_rows */
	void* stage_keys = nullptr;      /* materialised packed keys */
	void* stage_pay = nullptr;       /* materialised packed payloads */
	unsigned long long* words = nullptr; /* [0] materialised count, [1] bucket mask */
	int64_t max_buckets = 0;
	bool direct = false;             /* build inserts directly into a table sized for build_rows */
	uint64_t direct_bmask = 0;       /* bucket mask of the direct table */
	size_t table_bytes = 0;
	bool dense = false;              /* direct-address table indexed by the packed key */
	int slot_bytes() const { return (key64 || pay64) ? 16 : 8; }
	/* entry width of a dense table: 0 = bitmap (no payload), else 4 or 8 bytes of payload + 1 */
	int dense_entry_bytes() const { return pay_bits == 0 ? 0 : (pay_bits <= 31 ? 4 : 8); }
};

struct Op {
	enum Kind { Filter, Probe } kind;
	BExprP pred;                 /* Filter */
	int join = -1;               /* Probe: index into LoweredPlan::joins */
	std::vector<BExprP> keys;    /* Probe keys */
	int npay = 0;                /* Probe: payload outputs */
};

struct Sink {
	enum Kind { JoinBuild, AggGlobal, AggDense, AggHash, Emit } kind;
	int join = -1;
	std::vector<BExprP> keys;    /* build keys / group keys */
	std::vector<BExprP> pay;     /* build payloads */
	struct Agg {
		bool count = false;
		BExprP arg;
		bool visible = true;
	};
	std::vector<Agg> aggs;       /* group/global aggregates (+ hidden count) */
	int count_idx = -1;
	std::vector<BExprP> outs;    /* Emit columns */
	/* group key packing */
	std::vector<int> key_shift;
	std::vector<int64_t> key_radix;
	int key_bits = 0;
	__int128 domain = 0;         /* product of key ranges */
	int64_t groups_bound = 0;    /* upper bound of distinct groups */
	/* packed accumulator words of a hash group table: aggregate a's sum of (value - lower
	 * bound) -- the count for a count -- is the bit field [agg_shift[a], agg_shift[a] +
	 * agg_bits[a]) of word agg_word[a]; the bounds keep every field from carrying over */
	std::vector<int> agg_word, agg_shift, agg_bits;
	int nwords = 0;
};

/* An aggregation's result kept on the device as the input of a later pipeline of the same
 * query: the reference's bucket_flush + re-aggregation + read chain (relalg_translator.cpp
 * :659-809) becomes one table of int64 columns key_<i>, aggr_<j> with a device-side row
 * count, written by the producing pipeline's sink and scanned by the consumer. */
struct InterTable {
	std::string name;                 /* aggr_ht<N>, as the reference's translator names it */
	int producer = -1;                /* pipeline whose sink writes the rows */
	int64_t cap = 0;                  /* row capacity: the producer's groups bound */
	std::vector<Column> cols;         /* int64 columns with their value bounds */
	int64_t* out = nullptr;           /* cols x cap, column-major */
	unsigned long long* count = nullptr;
};

struct PipeColumn {
	std::string table, name;
	int type;
	int64_t lo, hi;
	bool host = false;        /* read from pinned host memory (coherent loads, no bulk copies) */
};

struct Pipeline {
	int id = 0;
	std::string table;
	int64_t rows = 0;
	std::vector<PipeColumn> cols;
	std::vector<Op> ops;
	Sink sink;
	int source_inter = -1;       /* scans an intermediate table (row count read on the device) */
	int out_inter = -1;          /* the sink writes an intermediate table, not the query result */
	int err_slot = -1;           /* parameter slot of the device error word */
	std::vector<int> col_slots;  /* parameter slots of the column pointers */
};

/* the tunable knobs of one CUDA flavor (the computation_type=cuda(...) blend) */
struct Flavor {
	int threads = 256;        /* threads per CTA */
	int rows = 4;             /* consecutive rows per thread and tile step */
	std::string aggr = "auto";/* auto | dense | global | cache | part */
	int cache_slots = 1024;   /* shared-memory group cache (aggr=cache) */
	int bucket = 32;          /* join bucket bytes: 32 (sector) or the slot size */
	int grid = 0;             /* CTAs per SM (0 = occupancy) */
	int dense_limit = 4096;   /* largest dense key domain */
	bool graph = true;        /* replay the query's launches from a CUDA graph */
	std::string load = "ldg"; /* column tiles: ldg (vector loads) | tma (bulk copies into a smem ring) */
	int stages = 4;           /* tma ring depth */
	std::string build = "auto"; /* join build: auto | direct | staged | dense */
	bool prefetch = true;     /* ldg: load the next tile while the current one is processed */
	std::string stream = "ldg"; /* column loads: ldg (read-only path) | noalloc (read-only path without
	                             * L1 allocation, so probed tables keep L1) */
	int compact = -2;         /* compact survivors after op k (-1 never, -2 auto) */
	std::string lowcard = "packed";  /* dense aggregation: combine (warp pre-sum by shuffles) | atomic (per-warp
	                                  * replicas) | private (per-thread accumulators behind a block dictionary)
	                                  * | redux (warp pre-sum by redux.sync into per-warp replicas) | regs
	                                  * (per-thread packed register accumulators behind a block dictionary,
	                                  * folded per warp every few tiles) | packed (the same packed words in
	                                  * shared memory, one column per thread); regs and packed run as
	                                  * combine where they do not apply (survivor compaction, joinN loops,
	                                  * batches, slots in global memory) */
	std::string hash = "mix"; /* table positions: mix (finalizer of the packed key) | voila (runtime.hpp hash) */
	int fill = 50;            /* largest load factor (percent) of group tables */
	int64_t direct_limit = 64ll << 20; /* auto: direct when the upper-bound table fits this many bytes */
	int sink_smem = 96 * 1024; /* most shared memory a dense aggregation keeps its slots in (else global) */
	int64_t group_slots = 0;  /* hash group table slots (0 = sized from the groups bound and fill) */
	int probe_lanes = 1;      /* lanes that probe one join key together (1 = each lane its own key) */
	int private_groups = 8;   /* lowcard=private|regs|packed: groups per CTA with per-thread accumulators */
	int min_ctas = 0;         /* CTAs per SM the main kernel's registers must allow (0 = no bound) */
	int flush_rows = 8;       /* compaction: survivors per thread and pass of a flush */
	int parts = 0;            /* aggr=part: partitions (0 = from the groups bound) */
	int64_t out_rows = 0;     /* result row capacity of an emitting pipeline (0 = from its bound, at
	                           * most 4 rows per input row + 2^20 when joinN probes multiply rows) */

	/* per-pipeline overrides "p<id>=cuda(...)" applied on top of these knobs (the reference's
	 * per-pipeline blends, QueryConfig::pipeline_default_blend) */
	std::vector<std::pair<int, std::string>> overrides;

	std::string str() const;
	static Flavor parse(const std::string& s);
	/* the knobs pipeline `id` runs with */
	Flavor for_pipe(int id) const;

private:
	static void apply(Flavor& f, const std::string& s);
};

/* A result column as the caller sees it: the sum of physical result-buffer columns, each
 * shifted left by its amount.  Every column has one part except a sum whose bound leaves
 * int64, which is computed as exact int64 sums of bit chunks and recombined in 128 bits. */
struct OutCol {
	std::vector<std::pair<int, int>> parts; /* (physical column, shift) */
	bool str = false;                       /* a string dictionary code, printed as its string */
};

/* Code set of a `contains` predicate: bit (code - lo) is set when the code's string holds the
 * pattern.  Uploaded at query creation; `dev` is its device copy. */
struct CodeBitmap {
	int64_t lo = 0;
	std::vector<uint32_t> bits;
	void* dev = nullptr;
};

struct LoweredPlan {
	std::vector<Pipeline> pipes;
	std::vector<JoinDesc> joins;
	std::vector<InterTable> inters;
	int result_pipe = -1;
	int result_cols = 0;              /* physical columns of the result buffer */
	std::vector<OutCol> out_cols;     /* the caller's columns */
	std::vector<CodeBitmap> bitmaps;  /* code sets of `contains` predicates */
};

LoweredPlan lower_plan(const RelOpP& root, std::map<std::string, Table>& tables, const Flavor& fl,
	const StringDict& dict);

/* ------------------------------------------------------------------ generated code ----- */

struct Launch {
	enum Kind { Kernel, MemsetZero } kind = Kernel;
	std::string kernel;
	int pipe = -1;
	int stage = 0;               /* which kernel of the pipeline */
	size_t smem = 0;
	int threads = 256;
	int64_t grid_items = 0;      /* work items that bound the grid (0 = persistent over SMs) */
	int64_t grid_cap = 0;        /* most CTAs (0 = no limit) */
	int grid_with = -1;          /* launch whose grid this one repeats (same tiles per CTA) */
	bool dominant = false;       /* the fact pipeline's main kernel */
	void** memset_ptr = nullptr; /* MemsetZero */
	size_t memset_bytes = 0;
};

struct GeneratedCode {
	std::string source;
	std::vector<Launch> launches;
};

/* device state of one pipeline's sink, allocated before code generation */
/* Partitioned hash aggregation of one pipeline (flavor aggr=part; voila_device.cuh describes
 * the two passes).  P == 0: the pipeline aggregates into a global group table instead. */
struct PartPlan {
	int P = 0;                 /* partitions (power of two) */
	int log2P = 0;
	int S = 0;                 /* slots of a partition's shared-memory table (power of two) */
	int rec_words = 1;         /* 64-bit words per record */
	std::vector<int> rec_word, rec_off; /* per aggregate: its record field (count: -1) */
	int agg_threads = 512;     /* threads of the aggregation kernel */
	int64_t cap = 0;           /* record capacity (below 2^32) */
	int64_t R = 0;             /* records above which a partition is split over several items */
	int64_t max_items = 0;
	int64_t scratch = 0;       /* capacity of the split partitions' partial groups */
	size_t smem1 = 0, smem2 = 0; /* dynamic shared memory of the two passes */
	int64_t max_ctas = 0;      /* most CTAs of the histogram and scatter passes */
	void* buf = nullptr;       /* records, partition after partition */
	void* cnt = nullptr;       /* max_ctas x P: the histogram pass's count per CTA and partition */
	void* skeys = nullptr;     /* partial groups: stored keys */
	void* sacc = nullptr;      /* partial groups: accumulator words */
	void* items = nullptr;     /* per split item: (scratch position << 16) | groups */
	unsigned long long* ctl = nullptr; /* per run: item counter, partial cursor, histogram done
	                                    * counter, P record totals, P starts, P scatter cursors,
	                                    * P split-item done counters (u32) */
};

/* the partitioned aggregation of pipeline p under flavor f, or P == 0 when it does not apply
 * (not a hash group-by, keys wider than 31 bits, records wider than 128 bits, ...) */
PartPlan part_plan(const Pipeline& p, const LoweredPlan& plan, const Flavor& f, int sms);

struct PipeDeviceState {
	void* sink_dev = nullptr;            /* aggregation state (global sums, dense slots, group table) */
	int64_t sink_cap = 0;
	size_t sink_bytes = 0;
	void* sink_acc = nullptr;            /* hash group table: accumulator words (sink_dev holds the keys) */
	bool sink_direct = false;            /* group table indexed by the packed key itself (no keys
	                                      * stored): sink_cap slots of accumulator words */
	bool self_cleaning = false;          /* the pipeline's last kernel leaves sink_dev zeroed */
	void* stage_hash = nullptr;          /* staged join build: materialised hashes */
	unsigned long long* done = nullptr;  /* last-block counter */
	PartPlan part;                       /* partitioned aggregation (aggr=part) */
};

/* query-wide device state the generated kernels write to */
struct QueryDeviceState {
	int64_t* out = nullptr;              /* result_cols x out_cap, column-major */
	int64_t out_cap = 0;
	unsigned long long* out_count = nullptr;
};

GeneratedCode generate_cuda(LoweredPlan& plan, const Flavor& fl, std::vector<PipeDeviceState>& st,
	const QueryDeviceState& qs, std::vector<std::vector<unsigned long long>>& params);

/* ------------------------------------------------------------------ JIT ---------------- */

struct JitModule {
	cudaLibrary_t lib = nullptr;
	std::map<std::string, cudaKernel_t> kernels;
};

std::shared_ptr<JitModule> jit_compile(const std::string& source, std::string* log_out);
std::string jit_cubin(const std::string& source, std::string* log_out);
const std::string& device_header_source();

/* ------------------------------------------------------------------ engine ------------- */

struct Engine {
	int device = 0;
	int sms = 0;
	bool offline = false;       /* code generation and compilation only, no device */
	uintptr_t fake_next = 0x100000;
	std::map<std::string, Table> tables;
	StringDict dict;
	std::mutex mu;
	~Engine();
};

struct Query {
	Engine* eng = nullptr;
	std::string plan_text;
	Flavor flavor;
	LoweredPlan plan;
	GeneratedCode code;
	std::shared_ptr<JitModule> mod;
	std::vector<void*> allocations;
	unsigned* err = nullptr;             /* device error word */
	unsigned long long* out_count = nullptr;
	int64_t* out = nullptr;              /* result_cols x out_cap, column-major */
	int64_t out_cap = 0;
	std::vector<std::vector<unsigned long long>> params; /* per pipeline */
	cudaStream_t stream = nullptr;
	bool profile = false;
	std::vector<cudaEvent_t> ev;         /* per launch begin/end when profiling */
	std::vector<float> last_ms;
	cudaGraphExec_t graph = nullptr;
	bool graph_profiled = false;         /* the graph records the profiling events */
	cudaStream_t graph_stream = nullptr;
	bool ran = false;
	bool dirty = false;                  /* self-cleaning state may be left set: clear before the next run */
	int64_t result_rows = -1;
	int64_t* result_host = nullptr;      /* column-major copy of the last result (pinned host memory) */
	size_t result_host_cap = 0;          /* int64 words allocated at result_host */
	~Query();
};

/* device-side bookkeeping of one query (kept beside Query so batches can reuse it) */
struct QueryState {
	std::vector<PipeDeviceState> pipes;
	std::vector<cudaKernel_t> kernels;
	std::vector<int> occupancy;
	std::vector<std::pair<void*, size_t>> memsets;
	/* state a run leaves clear by itself (self-cleaning group tables): cleared once, and again
	 * only before a run that follows a failed one; batches clear it on every run */
	std::vector<std::pair<void*, size_t>> clean_memsets;
};

QueryState& state_of(Query& q);
void* column_dev(Query& q, const PipeColumn& pc);
void alloc_group_table(Query& q, const Pipeline& p, PipeDeviceState& ps);

/* ------------------------------------------------------------------ batches ------------ */

/* One unit of work of the persistent batch kernel (layout shared with the device code). */
struct BatchItem {
	int32_t shape;          /* which generated item function runs it */
	int32_t dep;            /* done-counter that must reach dep_target first, -1 = none */
	int64_t params;         /* offset of the pipeline's parameters in the parameter pool */
	int64_t begin, end;     /* tile (or slot-group) range */
	int64_t nitems;         /* items of this pipeline stage (last-item publication) */
	int64_t dep_target;
	int32_t done;           /* done-counter incremented when the item finishes */
	int32_t finish;         /* query whose completion time this item may record, -1 = none */
};

struct Batch {
	Engine* eng = nullptr;
	std::vector<Query*> queries;
	Flavor flavor;
	std::string source;
	std::shared_ptr<JitModule> mod;
	cudaKernel_t kernel = nullptr;
	int occupancy = 0;
	int regs = 0;
	size_t smem = 0;
	int64_t nitems = 0;
	std::vector<BatchItem> host_items; /* the work queue as uploaded (for inspection) */
	std::vector<void*> allocations;
	BatchItem* items = nullptr;
	unsigned long long* counters = nullptr; /* [0] queue head, [1..] done counters */
	size_t counters_bytes = 0;
	unsigned long long* params = nullptr;
	unsigned long long* finish = nullptr;   /* per query: completion globaltimer ns; [n] = start */
	unsigned* err = nullptr;
	std::vector<std::pair<void*, size_t>> memsets;
	cudaGraphExec_t graph = nullptr;
	cudaStream_t stream = nullptr;
	int grid = 0;
	unsigned long long wait_ns = 2000000000ull; /* longest wait of an item on its dependency */
	std::vector<BatchItem> held;               /* original items replaced by vc_batch_hold_item */
	std::vector<int64_t> held_index;
	~Batch();
};

struct BatchCode {
	std::string source;
	size_t smem = 0;
	std::vector<BatchItem> items;
	std::vector<unsigned long long> params;
	std::vector<int64_t> query_params_begin; /* query i's parameters: [begin[i], begin[i + 1]) */
	int ncounters = 0;
};

BatchCode generate_batch(std::vector<Query*>& queries, const std::vector<Flavor>& flavors, int threads,
	int64_t tiles_per_item);

void query_prepare(Query& q);
void query_launch(Query& q, cudaStream_t stream);
void query_fetch(Query& q);
std::string query_result_text(Query& q);

} // namespace vc

#endif
