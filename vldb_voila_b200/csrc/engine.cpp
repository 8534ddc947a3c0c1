/*
 * Runtime of the CUDA flavor and the C ABI declared in include/voila_cuda.h.
 *
 * A query follows the reference's lifecycle (Compiler::_generate -> call_cxx_compiler ->
 * voila_query_new -> per repetition voila_query_reset + voila_query_run, compiler.cpp:343-533):
 * plan text is lowered into pipelines, the pipelines' device state is allocated, one CUDA
 * module is generated and compiled for the whole query, and each run launches the pipelines
 * in order on one stream (Query::run runs pipelines sequentially, runtime_framework.cpp:166-198;
 * here the parallelism is inside each kernel instead of tbb::parallel_for over threads).
 */
#include <algorithm>
#include <cinttypes>
#include <cstring>
#include <thread>
#include <functional>
#include <sstream>

#include "engine_internal.hpp"
#include "workloads.hpp"
#include "../../include/voila_cuda.h"

namespace vc {

/* AOT kernels (datagen.cu) */
cudaError_t launch_generate(void* out, const vc_gen_spec& spec, const double* zipf_cdf_dev, int64_t rows,
	cudaStream_t stream);

static thread_local std::string g_last_error;

static int64_t pow2_at_least(int64_t x)
{
	int64_t p = 1;
	while (p < x) {
		p <<= 1;
	}
	return p;
}

/* ------------------------------------------------------------------ flavor ------------- */

std::string Flavor::str() const
{
	std::ostringstream o;
	o << "cuda(threads=" << threads << ",rows=" << rows << ",load=" << load;
	if (load == "tma") {
		o << ",stages=" << stages;
	}
	else {
		o << ",prefetch=" << (prefetch ? 1 : 0);
	}
	o << ",compact=" << (compact == -2 ? std::string("auto") : std::to_string(compact));
	o << ",aggr=" << aggr << ",lowcard=" << lowcard << ",hash=" << hash << ",fill=" << fill << ",cache=" << cache_slots
	  << ",build=" << build
	  << ",grid=" << grid << ",dense=" << dense_limit << ",graph=" << (graph ? 1 : 0);
	if (sink_smem != 96 * 1024) {
		o << ",sinksmem=" << sink_smem;
	}
	if (group_slots) {
		o << ",gcap=" << group_slots;
	}
	if (out_rows) {
		o << ",ocap=" << out_rows;
	}
	if (probe_lanes != 1) {
		o << ",probe=" << probe_lanes;
	}
	if (flush_rows != 8) {
		o << ",frows=" << flush_rows;
	}
	if (min_ctas) {
		o << ",minctas=" << min_ctas;
	}
	if (stream != "ldg") {
		o << ",stream=" << stream;
	}
	if (private_groups != 8) {
		o << ",pgroups=" << private_groups;
	}
	if (parts) {
		o << ",parts=" << parts;
	}
	o << ")";
	for (auto& ov : overrides) {
		o << ";p" << ov.first << "=" << ov.second;
	}
	return o.str();
}

Flavor Flavor::parse(const std::string& s0)
{
	/* "cuda(...)" for every pipeline, then ";p<id>=cuda(...)" overrides for single pipelines */
	Flavor f;
	std::string s = s0;
	s.erase(std::remove_if(s.begin(), s.end(), ::isspace), s.end());
	std::vector<std::string> parts;
	std::stringstream ss(s);
	std::string part;
	while (std::getline(ss, part, ';')) {
		parts.push_back(part);
	}
	if (parts.empty()) {
		return f;
	}
	apply(f, parts[0]);
	for (size_t i = 1; i < parts.size(); i++) {
		const std::string& ov = parts[i];
		const size_t eq = ov.find('=');
		if (ov.size() < 3 || ov[0] != 'p' || eq == std::string::npos) {
			throw Error(1, "pipeline flavor overrides look like p<id>=cuda(...), got '" + ov + "'");
		}
		int id = -1;
		try {
			id = std::stoi(ov.substr(1, eq - 1));
		} catch (...) {
			throw Error(1, "bad pipeline id in '" + ov + "'");
		}
		const std::string body = ov.substr(eq + 1);
		Flavor probe = f;
		apply(probe, body); /* validates the knobs */
		if (body.find("hash=") != std::string::npos || body.find("graph=") != std::string::npos) {
			throw Error(1, "hash and graph are knobs of the whole query, not of one pipeline");
		}
		if (id < 0) {
			throw Error(1, "bad pipeline id in '" + ov + "'");
		}
		f.overrides.push_back({id, body});
	}
	return f;
}

Flavor Flavor::for_pipe(int id) const
{
	Flavor f = *this;
	f.overrides.clear();
	for (auto& ov : overrides) {
		if (ov.first == id) {
			apply(f, ov.second);
		}
	}
	return f;
}

void Flavor::apply(Flavor& f, const std::string& s0)
{
	std::string s = s0;
	if (s.empty() || s == "cuda" || s == "cuda()") {
		return;
	}
	if (s.rfind("computation_type=", 0) == 0) {
		s = s.substr(17);
	}
	if (s.rfind("cuda(", 0) != 0 || s.back() != ')') {
		throw Error(1, "flavor must look like cuda(key=value,...), got '" + s0 + "'");
	}
	std::stringstream ss(s.substr(5, s.size() - 6));
	std::string item;
	while (std::getline(ss, item, ',')) {
		if (item.empty()) {
			continue;
		}
		auto eq = item.find('=');
		if (eq == std::string::npos) {
			throw Error(1, "flavor item without '=': " + item);
		}
		std::string k = item.substr(0, eq), v = item.substr(eq + 1);
		auto num = [&](int lo, int hi) {
			int x = 0;
			try {
				x = std::stoi(v);
			} catch (...) {
				throw Error(1, "flavor " + k + " must be an integer");
			}
			if (x < lo || x > hi) {
				throw Error(1, "flavor " + k + " out of range");
			}
			return x;
		};
		if (k == "threads") {
			f.threads = num(32, 1024);
			if (f.threads % 32) {
				throw Error(1, "threads must be a multiple of 32");
			}
		} else if (k == "rows") {
			f.rows = num(1, 16);
			if (f.rows & (f.rows - 1)) {
				throw Error(1, "rows must be a power of two");
			}
		} else if (k == "aggr") {
			if (v != "auto" && v != "dense" && v != "global" && v != "cache" && v != "part" && v != "direct" &&
				v != "dcache") {
				throw Error(1, "aggr must be auto, dense, global, cache, part, direct or dcache");
			}
			f.aggr = v;
		} else if (k == "cache") {
			f.cache_slots = num(32, 8192);
		} else if (k == "grid") {
			f.grid = num(0, 64);
		} else if (k == "dense") {
			f.dense_limit = num(1, 1 << 22);
		} else if (k == "probe") {
			f.probe_lanes = num(1, 32);
			if (f.probe_lanes & (f.probe_lanes - 1)) {
				throw Error(1, "probe lanes must be a power of two");
			}
		} else if (k == "frows") {
			f.flush_rows = num(1, 16);
			if (f.flush_rows & (f.flush_rows - 1)) {
				throw Error(1, "frows must be 1, 2, 4, 8 or 16");
			}
		} else if (k == "pgroups") {
			f.private_groups = num(1, 16);
		} else if (k == "minctas") {
			f.min_ctas = num(0, 32);
		} else if (k == "stream") {
			if (v != "ldg" && v != "noalloc") {
				throw Error(1, "stream must be ldg or noalloc");
			}
			f.stream = v;
		} else if (k == "parts") {
			f.parts = num(0, 2048);
			if (f.parts && (f.parts < 16 || (f.parts & (f.parts - 1)))) {
				throw Error(1, "parts must be 0 or a power of two from 16 to 2048");
			}
		} else if (k == "ocap") {
			f.out_rows = num(0, 1 << 30);
		} else if (k == "gcap") {
			f.group_slots = num(0, 1 << 30);
		} else if (k == "sinksmem") {
			f.sink_smem = num(0, 96 * 1024);
		} else if (k == "graph") {
			f.graph = num(0, 1) != 0;
		} else if (k == "load") {
			if (v != "ldg" && v != "tma") {
				throw Error(1, "load must be ldg or tma");
			}
			f.load = v;
		} else if (k == "stages") {
			f.stages = num(2, 8);
		} else if (k == "prefetch") {
			f.prefetch = num(0, 1) != 0;
		} else if (k == "compact") {
			f.compact = v == "auto" ? -2 : num(-1, 64);
		} else if (k == "lowcard") {
			if (v != "combine" && v != "atomic" && v != "private" && v != "redux" && v != "regs" && v != "packed") {
				throw Error(1, "lowcard must be combine, atomic, private, redux, regs or packed");
			}
			f.lowcard = v;
		} else if (k == "hash") {
			if (v != "mix" && v != "voila") {
				throw Error(1, "hash must be mix or voila");
			}
			f.hash = v;
		} else if (k == "fill") {
			f.fill = num(10, 90);
		} else if (k == "build") {
			if (v != "auto" && v != "direct" && v != "staged" && v != "dense") {
				throw Error(1, "build must be auto, direct, staged or dense");
			}
			f.build = v;
		} else {
			throw Error(1, "unknown flavor knob '" + k + "'");
		}
	}
}

/* ------------------------------------------------------------------ engine ------------- */

Engine::~Engine()
{
	if (offline) {
		return;
	}
	cudaSetDevice(device);
	for (auto& t : tables) {
		for (auto& c : t.second.cols) {
			if (c.owned && c.dev) {
				cudaFree(c.dev);
			}
		}
	}
}

static void* dev_alloc(Query& q, size_t bytes)
{
	void* p = nullptr;
	if (q.eng->offline) {
		/* stand-in addresses: offline engines only generate and compile code */
		p = (void*)q.eng->fake_next;
		q.eng->fake_next += ((bytes + 255) / 256 + 1) * 256;
		return p;
	}
	/* whole 256-byte granules: bulk clears may round a region up to 16 bytes */
	VC_CHECK_CUDA(cudaMalloc(&p, std::max<size_t>((bytes + 255) & ~(size_t)255, 256)));
	q.allocations.push_back(p);
	return p;
}

Query::~Query()
{
	if (eng && eng->offline) {
		return;
	}
	if (eng) {
		cudaSetDevice(eng->device);
	}
	if (graph) {
		cudaGraphExecDestroy(graph);
	}
	for (auto e : ev) {
		cudaEventDestroy(e);
	}
	for (void* p : allocations) {
		cudaFree(p);
	}
	if (result_host) {
		cudaFreeHost(result_host);
	}
}

static std::map<Query*, QueryState> g_state;
QueryState& state_of(Query& q);

/* A batch runs a partitioned group-by (aggr=part) through the global split group table
 * instead: allocated here on first use (keys in 32-byte buckets, then the packed accumulator
 * words) and cleared once; the batch clears it before every run. */
void alloc_group_table(Query& q, const Pipeline& p, PipeDeviceState& ps)
{
	const Flavor pf = q.flavor.for_pipe(p.id);
	const int fill = pf.fill;
	ps.sink_cap = pf.group_slots > 0 ? pow2_at_least(pf.group_slots)
		: std::max<int64_t>(pow2_at_least((std::max<int64_t>(p.sink.groups_bound, 1) * 100 + fill - 1) / fill), 1024);
	const size_t kb = (((size_t)ps.sink_cap * (p.sink.key_bits <= 31 ? 4 : 8)) + 255) & ~(size_t)255;
	ps.sink_bytes = kb + (size_t)ps.sink_cap * p.sink.nwords * 8;
	ps.sink_dev = dev_alloc(q, ps.sink_bytes);
	ps.sink_acc = (char*)ps.sink_dev + kb;
	if (!q.eng->offline) {
		ps.self_cleaning = true;
		VC_CHECK_CUDA(cudaMemset(ps.sink_dev, 0, ps.sink_bytes));
		state_of(q).clean_memsets.push_back({ps.sink_dev, ps.sink_bytes});
	}
}
static std::mutex g_state_mu;

QueryState& state_of(Query& q)
{
	std::lock_guard<std::mutex> g(g_state_mu);
	return g_state[&q];
}

/* device data of a pipeline column: a base table's column or an intermediate table's */
void* column_dev(Query& q, const PipeColumn& pc)
{
	for (auto& it : q.plan.inters) {
		if (it.name == pc.table) {
			for (auto& c : it.cols) {
				if (c.name == pc.name) {
					return c.dev;
				}
			}
			return nullptr;
		}
	}
	Column* col = q.eng->tables.at(pc.table).find(pc.name);
	return col ? col->dev : nullptr;
}

void query_prepare(Query& q)
{
	Engine& e = *q.eng;
	if (!e.offline) {
		VC_CHECK_CUDA(cudaSetDevice(e.device));
	}
	RelOpP root = parse_plan(q.plan_text);
	q.plan = lower_plan(root, e.tables, q.flavor, e.dict);
	LoweredPlan& plan = q.plan;
	QueryState& st = state_of(q);
	st.pipes.assign(plan.pipes.size(), PipeDeviceState());

	/* Small per-run state (error word, result count, last-block counters, join counters,
	 * global and small dense accumulators) lives in one arena cleared by one memset. */
	const size_t arena_cap = 1 << 20;
	char* arena = (char*)dev_alloc(q, arena_cap);
	size_t arena_used = 0;
	auto arena_take = [&](size_t bytes) -> void* {
		size_t off = (arena_used + 255) & ~(size_t)255;
		if (off + bytes > arena_cap) {
			return nullptr;
		}
		arena_used = off + bytes;
		return arena + off;
	};
	q.err = (unsigned*)arena_take(8);
	q.out_count = (unsigned long long*)arena_take(8);
	/* code sets of `contains` predicates */
	for (auto& bm : plan.bitmaps) {
		const size_t bytes = bm.bits.size() * sizeof(uint32_t);
		bm.dev = dev_alloc(q, bytes);
		if (!e.offline) {
			VC_CHECK_CUDA(cudaMemcpy(bm.dev, bm.bits.data(), bytes, cudaMemcpyHostToDevice));
		}
	}

	for (auto& jd : plan.joins) {
		const int64_t rows = std::max<int64_t>(jd.build_rows, 1);
		const int sb = jd.slot_bytes();
		const int spb = std::max(1, 32 / sb);
		const int64_t slots = std::max<int64_t>(pow2_at_least(2 * rows), 2 * spb);
		jd.max_buckets = slots / spb;
		jd.table_bytes = (size_t)slots * sb;
		/* the build pipeline's knobs size its table */
		int build_pipe = 0;
		for (auto& p : plan.pipes) {
			if (p.sink.kind == Sink::JoinBuild && p.sink.join == jd.id) {
				build_pipe = p.id;
			}
		}
		const Flavor jf = q.flavor.for_pipe(build_pipe);
		const std::string& bm = jf.build;
		/* a dense table when the packed key space is small: one access per probe and no
		 * larger than the hash table would be (a bitmap when there is no payload) */
		size_t dense_bytes = 0;
		if (jd.key_bits <= 30) {
			const uint64_t span = 1ull << jd.key_bits;
			const int eb = jd.dense_entry_bytes();
			dense_bytes = eb == 0 ? (size_t)std::max<uint64_t>((span + 31) / 32, 1) * 4 : (size_t)(span * eb);
			dense_bytes = (dense_bytes + 15) & ~(size_t)15;
		}
		if (bm == "dense" && dense_bytes == 0) {
			throw Error(VC_ERR_UNSUPPORTED, "build=dense needs a join key space of at most 2^30 values");
		}
		/* a dense table holds one entry per key: JoinN (duplicate build keys) needs the hash table */
		if (bm == "dense" && !jd.join01) {
			throw Error(VC_ERR_UNSUPPORTED, "build=dense cannot hold the duplicate keys of a joinN build");
		}
		jd.dense = jd.join01 && dense_bytes > 0 &&
			(bm == "dense" || (bm == "auto" && dense_bytes <= std::max<size_t>(jd.table_bytes, 1 << 20)));
		if (jd.dense) {
			jd.table_bytes = dense_bytes;
		}
		jd.direct = jd.dense || bm == "direct" || (bm == "auto" && (int64_t)jd.table_bytes <= jf.direct_limit);
		jd.direct_bmask = (uint64_t)(jd.max_buckets - 1);
		jd.table = dev_alloc(q, jd.table_bytes);
		jd.words = (unsigned long long*)arena_take(32);
		if (jd.direct) {
			st.memsets.push_back({jd.table, jd.table_bytes});
		} else {
			jd.stage_keys = dev_alloc(q, (size_t)rows * (jd.key64 ? 8 : 4));
			jd.stage_pay = dev_alloc(q, (size_t)rows * (jd.pay64 ? 8 : 4));
		}
	}
	/* intermediate tables: int64 columns of `cap` rows each, and a row count in the arena */
	for (auto& it : plan.inters) {
		it.out = (int64_t*)dev_alloc(q, (size_t)it.cap * it.cols.size() * 8);
		it.count = (unsigned long long*)arena_take(8);
		for (size_t c = 0; c < it.cols.size(); c++) {
			it.cols[c].dev = it.out + (size_t)c * it.cap;
		}
	}
	Pipeline& rp = plan.pipes[plan.result_pipe];
	for (auto& p : plan.pipes) {
		PipeDeviceState& ps = st.pipes[p.id];
		const int A = (int)p.sink.aggs.size();
		ps.done = (unsigned long long*)arena_take(8);
		switch (p.sink.kind) {
		case Sink::JoinBuild:
			if (!plan.joins[p.sink.join].direct) {
				ps.stage_hash = dev_alloc(q, (size_t)std::max<int64_t>(plan.joins[p.sink.join].build_rows, 1) * 8);
			}
			break;
		case Sink::AggGlobal:
			ps.sink_cap = 1;
			ps.sink_bytes = (size_t)A * 8;
			break;
		case Sink::AggDense:
			ps.sink_cap = (int64_t)p.sink.domain;
			ps.sink_bytes = (size_t)p.sink.domain * A * 8;
			break;
		case Sink::AggHash:
			{
				/* direct group table (aggr=direct|dcache, and aggr=auto where it is no larger
				 * than the hash table would be): slot = packed key, so it needs no stored keys
				 * and no probes; every packed key below the largest one has a slot */
				const Flavor pf = q.flavor.for_pipe(p.id);
				__int128 pkmax = 0;
				for (size_t k = 0; k < p.sink.keys.size(); k++) {
					pkmax += (p.sink.keys[k]->b.hi - p.sink.keys[k]->b.lo) << p.sink.key_shift[k];
				}
				const __int128 dbytes = (pkmax + 1) * p.sink.nwords * 8;
				const __int128 hbytes = (__int128)std::max<int64_t>(pow2_at_least((std::max<int64_t>(p.sink.groups_bound, 1) *
					100 + pf.fill - 1) / pf.fill), 1024) * ((p.sink.key_bits <= 31 ? 4 : 8) + p.sink.nwords * 8);
				const bool want = pf.aggr == "direct" || pf.aggr == "dcache" ||
					(pf.aggr == "auto" && pf.group_slots == 0 && dbytes <= std::max<__int128>(hbytes, (__int128)16 << 20));
				/* a key space of 2^28 slots and more takes the hash table (aggr=dcache: behind
				 * the same shared-memory cache) */
				if (want && pkmax < ((__int128)1 << 28)) {
					ps.sink_direct = true;
					ps.sink_cap = (int64_t)pkmax + 1;
					ps.sink_bytes = (size_t)ps.sink_cap * p.sink.nwords * 8;
					break;
				}
			}
			ps.part = part_plan(p, plan, q.flavor.for_pipe(p.id), e.sms);
			if (ps.part.P > 0) {
				/* partitioned aggregation: records, partial groups of split partitions and
				 * per-item runs; its per-run counters live in the arena */
				PartPlan& pp = ps.part;
				pp.buf = dev_alloc(q, (size_t)pp.cap * 8 * pp.rec_words);
				pp.cnt = dev_alloc(q, (size_t)pp.max_ctas * pp.P * 4);
				pp.skeys = dev_alloc(q, (size_t)pp.scratch * 4);
				pp.sacc = dev_alloc(q, (size_t)pp.scratch * p.sink.nwords * 8);
				pp.items = dev_alloc(q, (size_t)pp.max_items * 8);
				pp.ctl = (unsigned long long*)arena_take(32 + (size_t)pp.P * 28);
				if (!pp.ctl) {
					throw Error(VC_ERR_UNSUPPORTED, "aggr=part: too many partitions for the per-run state");
				}
				break;
			}
			/* a user-set capacity (gcap) is taken as given: too small a table fails the run
			 * with VC_ERR_CAPACITY (bounded probe sequences), it never returns wrong rows */
			{
				const Flavor pf = q.flavor.for_pipe(p.id);
				ps.sink_cap = pf.group_slots > 0 ? pow2_at_least(pf.group_slots)
					: std::max<int64_t>(pow2_at_least((std::max<int64_t>(p.sink.groups_bound, 1) * 100 + pf.fill - 1) /
						pf.fill), 1024);
			}
			/* split layout: the keys (4 or 8 bytes per slot) in 32-byte buckets, then the
			 * packed accumulator words */
			ps.sink_bytes = (size_t)ps.sink_cap * (p.sink.key_bits <= 31 ? 4 : 8);
			ps.sink_bytes = (ps.sink_bytes + 255) & ~(size_t)255;
			ps.sink_bytes += (size_t)ps.sink_cap * p.sink.nwords * 8;
			break;
		case Sink::Emit:
			break;
		}
		if (ps.sink_bytes) {
			ps.sink_dev = ps.sink_bytes <= (64 << 10) ? arena_take(ps.sink_bytes) : nullptr;
			if (!ps.sink_dev) {
				ps.sink_dev = dev_alloc(q, ps.sink_bytes);
				if (p.sink.kind == Sink::AggHash && !e.offline) {
					/* the group extraction zeroes every slot it reads, so the table is left
					 * clear for the next run: it is cleared once here, not on every run
					 * (batches, which may skip items, still clear it per run) */
					ps.self_cleaning = true;
					VC_CHECK_CUDA(cudaMemset(ps.sink_dev, 0, ps.sink_bytes));
					st.clean_memsets.push_back({ps.sink_dev, ps.sink_bytes});
				} else {
					st.memsets.push_back({ps.sink_dev, ps.sink_bytes});
				}
			}
		}
		if (p.sink.kind == Sink::AggHash && ps.sink_direct) {
			ps.sink_acc = ps.sink_dev;
		} else if (p.sink.kind == Sink::AggHash && ps.part.P == 0) {
			const size_t kb = (((size_t)ps.sink_cap * (p.sink.key_bits <= 31 ? 4 : 8)) + 255) & ~(size_t)255;
			ps.sink_acc = (char*)ps.sink_dev + kb;
		}
	}
	st.memsets.insert(st.memsets.begin(), {arena, arena_used});
	switch (rp.sink.kind) {
	case Sink::AggGlobal: q.out_cap = 1; break;
	case Sink::AggDense: q.out_cap = (int64_t)rp.sink.domain; break;
	default:
		q.out_cap = std::max<int64_t>(rp.sink.groups_bound, 1);
		if (rp.sink.kind == Sink::Emit) {
			/* joinN can multiply rows up to probe rows x build rows: the buffer is bounded, and a
			 * result beyond it fails the run with VC_ERR_CAPACITY (raise it with ocap=) */
			const int64_t orows = q.flavor.for_pipe(rp.id).out_rows;
			const int64_t cap = orows > 0 ? orows : 4 * rp.rows + (1 << 20);
			q.out_cap = std::max<int64_t>(std::min(q.out_cap, cap), 1);
		}
		break;
	}
	q.out = (int64_t*)dev_alloc(q, (size_t)q.out_cap * plan.result_cols * 8);

	QueryDeviceState qs;
	qs.out = q.out;
	qs.out_cap = q.out_cap;
	qs.out_count = q.out_count;
	q.code = generate_cuda(plan, q.flavor, st.pipes, qs, q.params);
	/* a flavor whose shared memory (TMA ring + sink) exceeds the per-CTA opt-in limit is
	 * rejected here rather than failing at launch */
	int smem_optin = 232448; /* sm_100 */
	if (!e.offline) {
		VC_CHECK_CUDA(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, e.device));
	}
	for (auto& l : q.code.launches) {
		if (l.smem + 1024 > (size_t)smem_optin) {
			throw Error(VC_ERR_UNSUPPORTED, "flavor needs " + std::to_string(l.smem) + " bytes of shared memory per CTA in " +
				l.kernel + "; the device allows " + std::to_string(smem_optin));
		}
	}
	std::string log;
	if (e.offline) {
		jit_cubin(q.code.source, &log);
		return;
	}
	q.mod = jit_compile(q.code.source, &log);

	st.kernels.clear();
	st.occupancy.clear();
	for (auto& l : q.code.launches) {
		cudaKernel_t k;
		VC_CHECK_CUDA(cudaLibraryGetKernel(&k, q.mod->lib, l.kernel.c_str()));
		if (l.smem > 0) {
			/* static + dynamic shared memory above 48 KiB needs the opt-in.  Queries of one
			 * shape share this kernel with different (runtime-sized) shared memory, so the
			 * limit only ever grows. */
			cudaFuncAttributes fa;
			VC_CHECK_CUDA(cudaFuncGetAttributes(&fa, (const void*)k));
			if ((size_t)fa.maxDynamicSharedSizeBytes < l.smem) {
				VC_CHECK_CUDA(cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)l.smem));
			}
		}
		int occ = 0;
		VC_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, (const void*)k, l.threads, l.smem));
		if (occ < 1) {
			throw Error(6, "kernel " + l.kernel + " cannot be resident with its shared memory");
		}
		st.kernels.push_back(k);
		st.occupancy.push_back(occ);
	}
	/* fixed parameter slots: error word and column pointers */
	for (auto& p : plan.pipes) {
		auto& prm = q.params[p.id];
		prm[p.err_slot] = (unsigned long long)(uintptr_t)q.err;
		for (size_t c = 0; c < p.cols.size(); c++) {
			prm[p.col_slots[c]] = (unsigned long long)(uintptr_t)column_dev(q, p.cols[c]);
		}
	}
}

static void refresh_column_params(Query& q)
{
	for (auto& p : q.plan.pipes) {
		auto& prm = q.params[p.id];
		for (size_t c = 0; c < p.cols.size(); c++) {
			void* dev = column_dev(q, p.cols[c]);
			if (!dev) {
				throw Error(1, "column " + p.cols[c].table + "." + p.cols[c].name + " has no data");
			}
			prm[p.col_slots[c]] = (unsigned long long)(uintptr_t)dev;
		}
	}
}

static void launch_all(Query& q, cudaStream_t stream, bool capturing = false)
{
	QueryState& st = state_of(q);
	for (auto& m : st.memsets) {
		VC_CHECK_CUDA(cudaMemsetAsync(m.first, 0, m.second, stream));
	}
	const size_t n = q.code.launches.size();
	if (q.profile && q.ev.size() != 2 * n) {
		for (auto e : q.ev) {
			cudaEventDestroy(e);
		}
		q.ev.assign(2 * n, nullptr);
		for (auto& e : q.ev) {
			VC_CHECK_CUDA(cudaEventCreate(&e));
		}
	}
	std::vector<int64_t> grids(n, 1);
	for (size_t i = 0; i < n; i++) {
		const Launch& l = q.code.launches[i];
		const int g = q.flavor.for_pipe(l.pipe).grid;
		int occ = st.occupancy[i];
		if (l.grid_with >= 0) {
			/* the same tiles per CTA as the launch it repeats: the smaller occupancy of both */
			occ = std::min(occ, st.occupancy[(size_t)l.grid_with]);
		}
		for (size_t j = 0; j < n; j++) {
			if (q.code.launches[j].grid_with == (int)i) {
				occ = std::min(occ, st.occupancy[j]);
			}
		}
		int64_t per_sm = g > 0 ? std::min(g, occ) : occ;
		int64_t grid = (int64_t)q.eng->sms * per_sm;
		if (l.grid_items > 0) {
			grid = std::min<int64_t>(grid, l.grid_items);
		}
		if (l.grid_cap > 0) {
			grid = std::min<int64_t>(grid, l.grid_cap);
		}
		grids[i] = std::max<int64_t>(grid, 1);
	}
	for (size_t i = 0; i < n; i++) {
		const Launch& l = q.code.launches[i];
		const int64_t grid = l.grid_with >= 0 ? grids[(size_t)l.grid_with] : grids[i];
		void* args[] = {q.params[l.pipe].data()};
		if (q.profile) {
			VC_CHECK_CUDA(cudaEventRecordWithFlags(q.ev[2 * i], stream, capturing ? cudaEventRecordExternal : 0));
		}
		if (i > 0 && !q.profile) {
			/* programmatic dependent launch: this kernel is scheduled while the previous one
			 * finishes and waits (vd::pdl_wait) before touching what that one wrote */
			cudaLaunchConfig_t cfg = {};
			cfg.gridDim = dim3((unsigned)grid);
			cfg.blockDim = dim3((unsigned)l.threads);
			cfg.dynamicSmemBytes = l.smem;
			cfg.stream = stream;
			cudaLaunchAttribute attr[1];
			attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
			attr[0].val.programmaticStreamSerializationAllowed = 1;
			cfg.attrs = attr;
			cfg.numAttrs = 1;
			VC_CHECK_CUDA(cudaLaunchKernelExC(&cfg, (const void*)st.kernels[i], args));
		} else {
			VC_CHECK_CUDA(cudaLaunchKernel((const void*)st.kernels[i], dim3((unsigned)grid), dim3((unsigned)l.threads),
				args, l.smem, stream));
		}
		if (q.profile) {
			VC_CHECK_CUDA(cudaEventRecordWithFlags(q.ev[2 * i + 1], stream, capturing ? cudaEventRecordExternal : 0));
		}
	}
}

void query_launch(Query& q, cudaStream_t stream)
{
	if (q.eng->offline) {
		throw Error(7, "an offline engine only generates and compiles code");
	}
	VC_CHECK_CUDA(cudaSetDevice(q.eng->device));
	refresh_column_params(q);
	q.stream = stream;
	q.result_rows = -1;
	if (q.dirty) {
		for (auto& m : state_of(q).clean_memsets) {
			VC_CHECK_CUDA(cudaMemsetAsync(m.first, 0, m.second, stream));
		}
		q.dirty = false;
	}
	if (q.flavor.graph) {
		if (q.graph && q.graph_profiled != q.profile) {
			/* profiling events are nodes of the graph: re-capture when profiling toggles */
			cudaGraphExecDestroy(q.graph);
			q.graph = nullptr;
		}
		if (q.profile && q.ev.size() != 2 * q.code.launches.size()) {
			for (auto e : q.ev) {
				cudaEventDestroy(e);
			}
			q.ev.assign(2 * q.code.launches.size(), nullptr);
			for (auto& e : q.ev) {
				VC_CHECK_CUDA(cudaEventCreate(&e));
			}
		}
		if (!q.graph) {
			q.graph_profiled = q.profile;
			cudaStream_t cs;
			VC_CHECK_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
			cudaGraph_t g;
			VC_CHECK_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
			try {
				launch_all(q, cs, true);
			} catch (...) {
				cudaStreamEndCapture(cs, &g);
				cudaStreamDestroy(cs);
				throw;
			}
			VC_CHECK_CUDA(cudaStreamEndCapture(cs, &g));
			VC_CHECK_CUDA(cudaGraphInstantiate(&q.graph, g, 0));
			cudaGraphDestroy(g);
			cudaStreamDestroy(cs);
		}
		VC_CHECK_CUDA(cudaGraphLaunch(q.graph, stream));
	} else {
		launch_all(q, stream);
	}
	VC_CHECK_CUDA(cudaGetLastError());
	q.ran = true;
}

void query_fetch(Query& q)
{
	if (!q.ran || q.eng->offline) {
		throw Error(1, "query has not been run");
	}
	if (q.result_rows >= 0) {
		return;
	}
	VC_CHECK_CUDA(cudaSetDevice(q.eng->device));
	VC_CHECK_CUDA(cudaStreamSynchronize(q.stream));
	unsigned err = 0;
	unsigned long long cnt = 0;
	VC_CHECK_CUDA(cudaMemcpy(&err, q.err, sizeof(err), cudaMemcpyDeviceToHost));
	VC_CHECK_CUDA(cudaMemcpy(&cnt, q.out_count, sizeof(cnt), cudaMemcpyDeviceToHost));
	if (err) {
		q.dirty = true; /* a failed run may leave its tables set */
	}
	if (err & 1u) {
		throw Error(3, "a device hash table ran out of slots");
	}
	if (err & 2u) {
		throw Error(4, "a bounded device wait gave up");
	}
	if (err) {
		throw Error(3, "device error bits " + std::to_string(err));
	}
	if ((int64_t)cnt > q.out_cap) {
		throw Error(3, "result has more rows than its buffer");
	}
	q.result_rows = (int64_t)cnt;
	if (q.profile) {
		q.last_ms.assign(q.code.launches.size(), 0.f);
		for (size_t i = 0; i < q.code.launches.size(); i++) {
			VC_CHECK_CUDA(cudaEventElapsedTime(&q.last_ms[i], q.ev[2 * i], q.ev[2 * i + 1]));
		}
	}
	/* the result columns land in a pinned staging buffer (kept and grown across runs): a
	 * pageable destination would take the driver's slower staged copy */
	const int C = q.plan.result_cols;
	const size_t words = std::max<size_t>((size_t)C * cnt, 1);
	if (words > q.result_host_cap) {
		if (q.result_host) {
			VC_CHECK_CUDA(cudaFreeHost(q.result_host));
			q.result_host = nullptr;
			q.result_host_cap = 0;
		}
		VC_CHECK_CUDA(cudaMallocHost((void**)&q.result_host, words * 8));
		q.result_host_cap = words;
	}
	if (cnt > 0 && (int64_t)cnt == q.out_cap) {
		VC_CHECK_CUDA(cudaMemcpy(q.result_host, q.out, (size_t)C * cnt * 8, cudaMemcpyDeviceToHost));
	} else if (cnt > 0) {
		VC_CHECK_CUDA(cudaMemcpy2D(q.result_host, cnt * 8, q.out, (size_t)q.out_cap * 8, cnt * 8, (size_t)C,
			cudaMemcpyDeviceToHost));
	}
}

/* decimal text of a 128-bit integer */
static void append_i128(std::string& s, __int128 v)
{
	char buf[48];
	if (v >= (__int128)INT64_MIN && v <= (__int128)INT64_MAX) {
		const int len = std::snprintf(buf, sizeof(buf), "%" PRId64, (int64_t)v);
		s.append(buf, (size_t)len);
		return;
	}
	const bool neg = v < 0;
	unsigned __int128 u = neg ? (unsigned __int128)(-(v + 1)) + 1u : (unsigned __int128)v;
	int i = 47;
	buf[i] = 0;
	while (u) {
		buf[--i] = (char)('0' + (int)(u % 10u));
		u /= 10u;
	}
	if (neg) {
		buf[--i] = '-';
	}
	s.append(buf + i);
}

/* value of the caller's column c at row r: its physical parts, shifted and summed */
static __int128 result_value(const Query& q, int c, int64_t r)
{
	const int64_t R = q.result_rows;
	__int128 v = 0;
	for (auto& pt : q.plan.out_cols[(size_t)c].parts) {
		v += (__int128)q.result_host[(size_t)pt.first * R + r] * ((__int128)1 << pt.second);
	}
	return v;
}

std::string query_result_text(Query& q)
{
	query_fetch(q);
	const int C = (int)q.plan.out_cols.size();
	const int64_t R = q.result_rows;
	std::string s;
	s.reserve((size_t)R * C * 12);
	for (int64_t r = 0; r < R; r++) {
		for (int c = 0; c < C; c++) {
			if (c) {
				s.push_back('|');
			}
			const __int128 v = result_value(q, c, r);
			if (q.plan.out_cols[(size_t)c].str) {
				if (v < 0 || v >= (__int128)q.eng->dict.strings.size()) {
					throw Error(3, "a string result holds an unknown dictionary code");
				}
				s += q.eng->dict.strings[(size_t)v];
			} else {
				append_i128(s, v);
			}
		}
		s.push_back('\n');
	}
	return s;
}

/* the caller's columns as int64, column-major; a value beyond int64 is an error */
void query_result_int64(Query& q, int64_t* out, int64_t cap)
{
	query_fetch(q);
	const int64_t R = q.result_rows;
	const int C = (int)q.plan.out_cols.size();
	if (R * C > cap) {
		throw Error(1, "result buffer too small");
	}
	for (int c = 0; c < C; c++) {
		const auto& parts = q.plan.out_cols[(size_t)c].parts;
		if (parts.size() == 1 && parts[0].second == 0) {
			/* a plain int64 column: copied as is (large columns by several threads) */
			char* dst = (char*)(out + (size_t)c * R);
			const char* src = (const char*)(q.result_host + (size_t)parts[0].first * R);
			const size_t bytes = (size_t)R * 8;
			const size_t nt = std::min<size_t>(8, std::max<size_t>(1, bytes >> 22));
			if (nt == 1) {
				std::memcpy(dst, src, bytes);
				continue;
			}
			std::vector<std::thread> th;
			const size_t chunk = (bytes / nt + 63) & ~(size_t)63;
			for (size_t t = 0; t < nt; t++) {
				const size_t b = t * chunk;
				if (b < bytes) {
					th.emplace_back([=] { std::memcpy(dst + b, src + b, std::min(chunk, bytes - b)); });
				}
			}
			for (auto& x : th) {
				x.join();
			}
			continue;
		}
		for (int64_t r = 0; r < R; r++) {
			const __int128 v = result_value(q, c, r);
			if (v < (__int128)INT64_MIN || v > (__int128)INT64_MAX) {
				throw Error(3, "a result value exceeds int64: read it with vc_query_result_text");
			}
			out[(size_t)c * R + r] = (int64_t)v;
		}
	}
}

} // namespace vc

/* ====================================================================== C ABI ======== */

using namespace vc;

struct vc_engine {
	Engine e;
};
struct vc_query {
	Query q;
};

template <typename F>
static int guarded(F&& f)
{
	try {
		f();
		g_last_error.clear();
		return VC_OK;
	} catch (const Error& e) {
		g_last_error = e.what();
		return e.code;
	} catch (const std::bad_alloc&) {
		g_last_error = "out of host memory";
		return VC_ERR_INVALID;
	} catch (const std::exception& e) {
		g_last_error = e.what();
		return VC_ERR_INVALID;
	}
}

namespace vc {
/* status-code guard shared with the other translation units of the C ABI */
int abi_guard_mlp(const std::function<void()>& f)
{
	return guarded(f);
}

Query* vc_query_internal(vc_query* q)
{
	return &q->q;
}

/* the query's kernels ran inside a batch on stream s: results are read as after vc_query_run */
void query_mark_external_run(Query& q, cudaStream_t s)
{
	q.stream = s;
	q.ran = true;
	q.result_rows = -1;
	q.profile = false;
	q.dirty = false; /* the batch clears every table of the query before using it */
}
} // namespace vc

static int copy_out(const std::string& s, char* buf, size_t cap, size_t* len)
{
	if (len) {
		*len = s.size();
	}
	if (buf && cap) {
		size_t n = std::min(cap - 1, s.size());
		std::memcpy(buf, s.data(), n);
		buf[n] = 0;
	}
	return VC_OK;
}

static Table& table_of(vc_engine* eng, const char* t)
{
	if (!eng || !t) {
		throw Error(VC_ERR_INVALID, "null engine or table name");
	}
	auto it = eng->e.tables.find(t);
	if (it == eng->e.tables.end()) {
		throw Error(VC_ERR_INVALID, std::string("unknown table '") + t + "'");
	}
	return it->second;
}

static Column& column_of(vc_engine* eng, const char* t, const char* c)
{
	Table& tb = table_of(eng, t);
	Column* col = c ? tb.find(c) : nullptr;
	if (!col) {
		throw Error(VC_ERR_INVALID, std::string("unknown column '") + t + "." + (c ? c : "(null)") + "'");
	}
	return *col;
}

namespace vc {
Engine& engine_of(vc_engine* e)
{
	return e->e;
}

/* Declares an imported table with its columns (domains as observed) and uploads the host
 * data synchronously (the import's host buffers are released when it returns).  On a
 * compile-only engine the columns get stand-in addresses and no data. */
void import_declare(Engine& e, const std::string& table, int64_t rows, const std::vector<std::string>& names,
	const std::vector<int>& types, const std::vector<int64_t>& lo, const std::vector<int64_t>& hi,
	const std::vector<const void*>& data)
{
	std::lock_guard<std::mutex> g(e.mu);
	if (e.tables.count(table)) {
		throw Error(VC_ERR_INVALID, "table '" + table + "' exists");
	}
	Table t;
	t.name = table;
	t.rows = rows;
	try {
		for (size_t i = 0; i < names.size(); i++) {
			Column c;
			c.name = names[i];
			c.type = types[i];
			c.lo = rows ? lo[i] : 0;
			c.hi = rows ? hi[i] : 0;
			const size_t bytes = (size_t)std::max<int64_t>(rows, 1) * vc_gen_type_size(c.type);
			if (e.offline) {
				c.dev = (void*)e.fake_next;
				e.fake_next += ((bytes + 255) / 256 + 1) * 256;
			} else {
				VC_CHECK_CUDA(cudaSetDevice(e.device));
				VC_CHECK_CUDA(cudaMalloc(&c.dev, ((bytes + 255) / 256) * 256));
				c.owned = true;
				t.cols.push_back(c);
				if (rows) {
					VC_CHECK_CUDA(cudaMemcpy(c.dev, data[i], (size_t)rows * vc_gen_type_size(c.type),
						cudaMemcpyHostToDevice));
				}
				continue;
			}
			t.cols.push_back(c);
		}
	} catch (...) {
		for (auto& c : t.cols) {
			if (c.owned && c.dev) {
				cudaFree(c.dev);
			}
		}
		throw;
	}
	e.tables[table] = t;
}
} // namespace vc

extern "C" {

const char* vc_last_error(void)
{
	return g_last_error.c_str();
}

const char* vc_version(void)
{
	return "voila-b200 0.1 (sm_100a)";
}

int vc_engine_create(int device, vc_engine** out)
{
	return guarded([&] {
		if (!out) {
			throw Error(VC_ERR_INVALID, "null output");
		}
		int n = 0;
		if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
			cudaGetLastError();
			throw Error(VC_ERR_NO_DEVICE, "no CUDA device is available");
		}
		if (device < 0 || device >= n) {
			throw Error(VC_ERR_INVALID, "device index out of range");
		}
		VC_CHECK_CUDA(cudaSetDevice(device));
		cudaDeviceProp prop;
		VC_CHECK_CUDA(cudaGetDeviceProperties(&prop, device));
		if (prop.major < 10) {
			throw Error(VC_ERR_NO_DEVICE, "the CUDA flavor is built for sm_100a (B200); device is sm_" +
				std::to_string(prop.major) + std::to_string(prop.minor));
		}
		auto* e = new vc_engine();
		e->e.device = device;
		e->e.sms = prop.multiProcessorCount;
		*out = e;
	});
}

int vc_engine_create_offline(int sms, vc_engine** out)
{
	return guarded([&] {
		if (!out || sms < 1) {
			throw Error(VC_ERR_INVALID, "bad arguments");
		}
		auto* e = new vc_engine();
		e->e.offline = true;
		e->e.sms = sms;
		*out = e;
	});
}

int vc_engine_destroy(vc_engine* eng)
{
	return guarded([&] { delete eng; });
}

int vc_table_create(vc_engine* eng, const char* table, int64_t rows)
{
	return guarded([&] {
		if (!eng || !table || !*table || rows < 0) {
			throw Error(VC_ERR_INVALID, "bad table arguments");
		}
		std::lock_guard<std::mutex> g(eng->e.mu);
		if (eng->e.tables.count(table)) {
			throw Error(VC_ERR_INVALID, std::string("table '") + table + "' exists");
		}
		Table t;
		t.name = table;
		t.rows = rows;
		eng->e.tables[table] = t;
	});
}

int vc_table_drop(vc_engine* eng, const char* table)
{
	return guarded([&] {
		Table& t = table_of(eng, table);
		cudaSetDevice(eng->e.device);
		for (auto& c : t.cols) {
			if (c.owned && c.dev) {
				cudaFree(c.dev);
			}
		}
		eng->e.tables.erase(table);
	});
}

int vc_column_add(vc_engine* eng, const char* table, const char* column, int type, int64_t lo, int64_t hi)
{
	return guarded([&] {
		Table& t = table_of(eng, table);
		if (!column || !*column || type < VC_U8 || type > VC_STR || lo > hi) {
			throw Error(VC_ERR_INVALID, "bad column arguments");
		}
		if (type == VC_STR) {
			lo = hi = 0; /* a string column's domain is its dictionary codes, set by its upload */
		}
		if (t.find(column)) {
			throw Error(VC_ERR_INVALID, std::string("column '") + column + "' exists");
		}
		const int64_t tmin = type == VC_U8 ? 0 : type == VC_I16 ? INT16_MIN : (type == VC_I32 || type == VC_STR) ? INT32_MIN
			: INT64_MIN;
		const int64_t tmax = type == VC_U8 ? 255 : type == VC_I16 ? INT16_MAX : (type == VC_I32 || type == VC_STR) ? INT32_MAX
			: INT64_MAX;
		if (lo < tmin || hi > tmax) {
			throw Error(VC_ERR_INVALID, "column domain does not fit its type");
		}
		Column c;
		c.name = column;
		c.type = type;
		c.lo = lo;
		c.hi = hi;
		const size_t bytes = (size_t)std::max<int64_t>(t.rows, 1) * vc_gen_type_size(type);
		if (eng->e.offline) {
			c.dev = (void*)eng->e.fake_next;
			eng->e.fake_next += ((bytes + 255) / 256 + 1) * 256;
		} else {
			VC_CHECK_CUDA(cudaSetDevice(eng->e.device));
			VC_CHECK_CUDA(cudaMalloc(&c.dev, ((bytes + 255) / 256) * 256));
			c.owned = true;
		}
		t.cols.push_back(c);
	});
}

int vc_column_info(vc_engine* eng, const char* table, const char* column, int32_t* type, int64_t* lo, int64_t* hi,
	int64_t* rows)
{
	return guarded([&] {
		Table& t = table_of(eng, table);
		Column& c = column_of(eng, table, column);
		if (type) *type = c.type;
		if (lo) *lo = c.lo;
		if (hi) *hi = c.hi;
		if (rows) *rows = t.rows;
	});
}

int vc_column_upload(vc_engine* eng, const char* table, const char* column, const void* host, int64_t rows,
	void* stream)
{
	return guarded([&] {
		Table& t = table_of(eng, table);
		Column& c = column_of(eng, table, column);
		if (!host || rows != t.rows) {
			throw Error(VC_ERR_INVALID, "upload must provide exactly the table's rows");
		}
		if (c.type == VC_STR) {
			throw Error(VC_ERR_INVALID, "string columns are uploaded with vc_column_upload_strings");
		}
		VC_CHECK_CUDA(cudaSetDevice(eng->e.device));
		if (rows) {
			VC_CHECK_CUDA(cudaMemcpyAsync(c.dev, host, (size_t)rows * vc_gen_type_size(c.type), cudaMemcpyHostToDevice,
				(cudaStream_t)stream));
		}
	});
}

namespace vc {
/* encodes a string column's rows into the engine dictionary and uploads the codes; the
 * column's domain becomes the codes' range */
static void upload_codes(Engine& e, Column& c, int64_t rows, const std::function<std::string(int64_t)>& row)
{
	std::vector<int32_t> codes((size_t)rows);
	int32_t lo = 0, hi = 0;
	{
		std::lock_guard<std::mutex> g(e.mu);
		for (int64_t r = 0; r < rows; r++) {
			codes[(size_t)r] = e.dict.encode(row(r));
			lo = r == 0 ? codes[(size_t)r] : std::min(lo, codes[(size_t)r]);
			hi = r == 0 ? codes[(size_t)r] : std::max(hi, codes[(size_t)r]);
		}
	}
	c.lo = lo;
	c.hi = hi;
	if (!e.offline && rows) {
		VC_CHECK_CUDA(cudaSetDevice(e.device));
		VC_CHECK_CUDA(cudaMemcpy(c.dev, codes.data(), (size_t)rows * 4, cudaMemcpyHostToDevice));
	}
}
} // namespace vc

int vc_column_upload_strings(vc_engine* eng, const char* table, const char* column, const char* bytes,
	const int64_t* offsets, int64_t rows)
{
	return guarded([&] {
		Table& t = table_of(eng, table);
		Column& c = column_of(eng, table, column);
		if (c.type != VC_STR || rows != t.rows || (rows && (!bytes || !offsets))) {
			throw Error(VC_ERR_INVALID, "a string upload needs a string column, its rows, bytes and rows+1 offsets");
		}
		for (int64_t r = 0; r < rows; r++) {
			if (offsets[r + 1] < offsets[r] || offsets[r] < 0) {
				throw Error(VC_ERR_INVALID, "string offsets must not decrease");
			}
		}
		upload_codes(eng->e, c, rows, [&](int64_t r) {
			return std::string(bytes + offsets[r], (size_t)(offsets[r + 1] - offsets[r]));
		});
	});
}

int vc_dict_size(vc_engine* eng, int64_t* n)
{
	return guarded([&] {
		if (!eng || !n) {
			throw Error(VC_ERR_INVALID, "null argument");
		}
		std::lock_guard<std::mutex> g(eng->e.mu);
		*n = (int64_t)eng->e.dict.strings.size();
	});
}

int vc_dict_string(vc_engine* eng, int64_t code, char* buf, size_t cap, size_t* len)
{
	return guarded([&] {
		if (!eng) {
			throw Error(VC_ERR_INVALID, "null engine");
		}
		std::lock_guard<std::mutex> g(eng->e.mu);
		if (code < 0 || code >= (int64_t)eng->e.dict.strings.size()) {
			throw Error(VC_ERR_INVALID, "no such string code");
		}
		copy_out(eng->e.dict.strings[(size_t)code], buf, cap, len);
	});
}

int vc_column_download(vc_engine* eng, const char* table, const char* column, void* host, int64_t rows,
	void* stream)
{
	return guarded([&] {
		Table& t = table_of(eng, table);
		Column& c = column_of(eng, table, column);
		if (!host || rows != t.rows) {
			throw Error(VC_ERR_INVALID, "download must take exactly the table's rows");
		}
		VC_CHECK_CUDA(cudaSetDevice(eng->e.device));
		if (rows) {
			VC_CHECK_CUDA(cudaMemcpyAsync(host, c.dev, (size_t)rows * vc_gen_type_size(c.type), cudaMemcpyDeviceToHost,
				(cudaStream_t)stream));
			VC_CHECK_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
		}
	});
}

int vc_column_attach(vc_engine* eng, const char* table, const char* column, void* device_ptr)
{
	return guarded([&] {
		Column& c = column_of(eng, table, column);
		if (!device_ptr || ((uintptr_t)device_ptr & 15u)) {
			throw Error(VC_ERR_INVALID, "attached column memory must be non-null and 16-byte aligned");
		}
		VC_CHECK_CUDA(cudaSetDevice(eng->e.device));
		if (c.owned && c.dev) {
			VC_CHECK_CUDA(cudaFree(c.dev));
		}
		c.dev = device_ptr;
		c.owned = false;
		c.host = false;
	});
}

int vc_column_attach_host(vc_engine* eng, const char* table, const char* column, const void* host_ptr)
{
	return guarded([&] {
		Column& c = column_of(eng, table, column);
		if (!host_ptr || ((uintptr_t)host_ptr & 15u)) {
			throw Error(VC_ERR_INVALID, "host column memory must be non-null and 16-byte aligned");
		}
		if (eng->e.offline) {
			throw Error(VC_ERR_NO_DEVICE, "an offline engine only generates and compiles code");
		}
		VC_CHECK_CUDA(cudaSetDevice(eng->e.device));
		cudaPointerAttributes pa;
		VC_CHECK_CUDA(cudaPointerGetAttributes(&pa, host_ptr));
		if (pa.type != cudaMemoryTypeHost) {
			throw Error(VC_ERR_INVALID, "host column memory must be pinned (cudaHostAlloc or cudaHostRegister)");
		}
		void* dev = nullptr;
		VC_CHECK_CUDA(cudaHostGetDevicePointer(&dev, const_cast<void*>(host_ptr), 0));
		if (c.owned && c.dev) {
			VC_CHECK_CUDA(cudaFree(c.dev));
		}
		c.dev = dev;
		c.owned = false;
		c.host = true;
	});
}

int vc_column_device_ptr(vc_engine* eng, const char* table, const char* column, void** out)
{
	return guarded([&] {
		Column& c = column_of(eng, table, column);
		if (!out) {
			throw Error(VC_ERR_INVALID, "null output");
		}
		*out = c.dev;
	});
}

int vc_column_generate(vc_engine* eng, const char* table, const char* column, int32_t kind, int64_t a, int64_t b,
	int64_t c, double s, uint64_t seed, const double* zipf_cdf, void* stream)
{
	return guarded([&] {
		Table& t = table_of(eng, table);
		Column& col = column_of(eng, table, column);
		vc_gen_spec spec;
		spec.kind = kind;
		spec.type = col.type;
		spec.a = a;
		spec.b = b;
		spec.c = c;
		spec.s = s;
		spec.seed = seed;
		spec.n = t.rows;
		if (kind < VC_GEN_UNIFORM || kind > VC_GEN_WORDS) {
			throw Error(VC_ERR_INVALID, "unknown generator kind");
		}
		if ((kind == VC_GEN_WORDS) != (col.type == VC_STR)) {
			throw Error(VC_ERR_INVALID, "string columns take the words generator, and only they do");
		}
		if (kind == VC_GEN_WORDS) {
			/* strings are made on the host and dictionary-encoded; the codes are uploaded */
			char buf[VC_GEN_STR_WIDTH];
			upload_codes(eng->e, col, t.rows, [&](int64_t r) {
				const int n = vc_gen_string(&spec, r, buf);
				return std::string(buf, (size_t)n);
			});
			return;
		}
		if ((kind == VC_GEN_DIV || kind == VC_GEN_MOD) && b <= 0) {
			throw Error(VC_ERR_INVALID, "generator divisor must be positive");
		}
		if (kind == VC_GEN_UNIFORM && (b < a || (__int128)b - a >= (__int128)INT64_MAX)) {
			throw Error(VC_ERR_INVALID, "uniform range must be non-empty and below 2^63");
		}
		const bool skew = kind == VC_GEN_ZIPF && s != 0.0;
		if (skew && (!zipf_cdf || b < 1)) {
			throw Error(VC_ERR_INVALID, "skewed Zipf generation needs the CDF table");
		}
		VC_CHECK_CUDA(cudaSetDevice(eng->e.device));
		double* dcdf = nullptr;
		if (skew) {
			VC_CHECK_CUDA(cudaMalloc(&dcdf, (size_t)b * sizeof(double)));
			VC_CHECK_CUDA(cudaMemcpyAsync(dcdf, zipf_cdf, (size_t)b * sizeof(double), cudaMemcpyHostToDevice,
				(cudaStream_t)stream));
		}
		cudaError_t rc = launch_generate(col.dev, spec, dcdf, t.rows, (cudaStream_t)stream);
		if (dcdf) {
			cudaStreamSynchronize((cudaStream_t)stream);
			cudaFree(dcdf);
		}
		VC_CHECK_CUDA(rc);
	});
}

int vc_gen_host(int32_t kind, int32_t type, int64_t a, int64_t b, int64_t c, double s, uint64_t seed, int64_t n,
	const double* zipf_cdf, int64_t begin, int64_t count, void* out)
{
	return guarded([&] {
		if (!out || count < 0 || begin < 0 || type < VC_U8 || type > VC_STR || (type == VC_STR) != (kind == VC_GEN_WORDS)) {
			throw Error(VC_ERR_INVALID, "bad generator arguments");
		}
		vc_gen_spec spec{kind, type, a, b, c, s, seed, n};
		if (type == VC_STR) {
			/* fixed-width rows of VC_GEN_STR_WIDTH bytes, NUL-padded */
			char* o = (char*)out;
			for (int64_t i = 0; i < count; i++) {
				char* row = o + (size_t)i * VC_GEN_STR_WIDTH;
				std::memset(row, 0, VC_GEN_STR_WIDTH);
				vc_gen_string(&spec, begin + i, row);
			}
			return;
		}
		for (int64_t i = 0; i < count; i++) {
			vc_gen_store(type, out, i, vc_gen_value(&spec, zipf_cdf, begin + i));
		}
	});
}

int vc_gen_zipf_cdf(double s, int64_t n, double* out)
{
	return guarded([&] {
		if (!out || n < 1) {
			throw Error(VC_ERR_INVALID, "bad zipf arguments");
		}
		vc_gen_build_zipf_cdf(s, n, out);
	});
}

int vc_workload_describe(const char* spec, char* buf, size_t cap, size_t* len)
{
	return guarded([&] {
		if (!spec) {
			throw Error(VC_ERR_INVALID, "null spec");
		}
		std::string d;
		try {
			d = vc_workload::describe(vc_workload::make(spec));
		} catch (const std::invalid_argument& e) {
			throw Error(VC_ERR_INVALID, e.what());
		}
		copy_out(d, buf, cap, len);
	});
}

int vc_plan_columns(const char* plan, char* buf, size_t cap, size_t* len)
{
	return guarded([&] {
		if (!plan) {
			throw Error(VC_ERR_INVALID, "null plan");
		}
		RelOpP root = parse_plan(plan);
		std::vector<std::pair<std::string, std::string>> seen;
		std::function<void(const RelOpP&)> walk = [&](const RelOpP& op) {
			if (!op) {
				return;
			}
			if (op->kind == RelOp::Scan) {
				for (auto& c : op->columns) {
					std::pair<std::string, std::string> k(op->table, c);
					if (std::find(seen.begin(), seen.end(), k) == seen.end()) {
						seen.push_back(k);
					}
				}
			}
			walk(op->left);
			walk(op->right);
		};
		walk(root);
		std::string d;
		for (auto& k : seen) {
			d += k.first + " " + k.second + "\n";
		}
		copy_out(d, buf, cap, len);
	});
}

int vc_workload_batch(int count, uint64_t seed, int64_t min_rows, int64_t max_rows, char* buf, size_t cap,
	size_t* len)
{
	return guarded([&] {
		if (count < 0 || min_rows < 1 || max_rows < min_rows) {
			throw Error(VC_ERR_INVALID, "bad batch arguments");
		}
		std::string s;
		for (auto& w : vc_workload::make_batch(count, seed, min_rows, max_rows)) {
			s += w + "\n";
		}
		copy_out(s, buf, cap, len);
	});
}

int vc_query_new(vc_engine* eng, const char* plan, const char* flavor, vc_query** out)
{
	vc_query* q = nullptr;
	int rc = guarded([&] {
		if (!eng || !plan || !out) {
			throw Error(VC_ERR_INVALID, "null argument");
		}
		q = new vc_query();
		q->q.eng = &eng->e;
		q->q.plan_text = plan;
		q->q.flavor = Flavor::parse(flavor ? flavor : "");
		query_prepare(q->q);
		*out = q;
	});
	if (rc != VC_OK && q) {
		std::string msg = g_last_error;
		{
			std::lock_guard<std::mutex> g(g_state_mu);
			g_state.erase(&q->q);
		}
		delete q;
		g_last_error = msg;
	}
	return rc;
}

int vc_query_run(vc_query* q, void* stream)
{
	return guarded([&] {
		if (!q) {
			throw Error(VC_ERR_INVALID, "null query");
		}
		query_launch(q->q, (cudaStream_t)stream);
	});
}

int vc_query_reset(vc_query* q)
{
	return guarded([&] {
		if (!q) {
			throw Error(VC_ERR_INVALID, "null query");
		}
		q->q.result_rows = -1;
	});
}

int vc_query_free(vc_query* q)
{
	return guarded([&] {
		if (q) {
			{
				std::lock_guard<std::mutex> g(g_state_mu);
				g_state.erase(&q->q);
			}
			delete q;
		}
	});
}

int vc_query_result_shape(vc_query* q, int64_t* rows, int32_t* cols)
{
	return guarded([&] {
		if (!q) {
			throw Error(VC_ERR_INVALID, "null query");
		}
		query_fetch(q->q);
		if (rows) {
			*rows = q->q.result_rows;
		}
		if (cols) {
			*cols = (int32_t)q->q.plan.out_cols.size();
		}
	});
}

int vc_query_result_copy(vc_query* q, int64_t* out, int64_t cap)
{
	return guarded([&] {
		if (!q || !out) {
			throw Error(VC_ERR_INVALID, "null argument");
		}
		query_result_int64(q->q, out, cap);
	});
}

int vc_query_result_text(vc_query* q, char* buf, size_t cap, size_t* len)
{
	return guarded([&] {
		if (!q) {
			throw Error(VC_ERR_INVALID, "null query");
		}
		copy_out(query_result_text(q->q), buf, cap, len);
	});
}

/* JSON list of a lowered plan's pipelines: what the flavor chooser featurizes */
static std::string describe_pipelines(const LoweredPlan& plan)
{
	static const char* sinks[] = {"join_build", "aggr_global", "aggr_dense", "aggr_hash", "emit"};
	std::ostringstream o;
	o << "[";
	for (size_t i = 0; i < plan.pipes.size(); i++) {
		auto& p = plan.pipes[i];
		int64_t bytes = 0;
		for (auto& c : p.cols) {
			bytes += p.rows * vc_gen_type_size(c.type);
		}
		int probes = 0, probes_n = 0, filters = 0;
		int64_t build_rows = 0;
		for (auto& op : p.ops) {
			if (op.kind == Op::Filter) {
				filters++;
			} else {
				probes++;
				probes_n += plan.joins[op.join].join01 ? 0 : 1;
				build_rows += plan.joins[op.join].build_rows;
			}
		}
		const double domain = p.sink.domain > 0 ? (double)p.sink.domain : 0.0;
		o << (i ? ", " : "") << "{\"table\": \"" << p.table << "\", \"rows\": " << p.rows << ", \"columns\": "
		  << p.cols.size() << ", \"ops\": " << p.ops.size() << ", \"filters\": " << filters << ", \"probes\": " << probes
		  << ", \"probes_n\": " << probes_n << ", \"probed_build_rows\": " << build_rows << ", \"sink\": \""
		  << sinks[p.sink.kind] << "\", \"aggregates\": " << p.sink.aggs.size() << ", \"key_domain\": " << domain
		  << ", \"groups_bound\": " << p.sink.groups_bound << ", \"scan_bytes\": " << bytes
		  << ", \"intermediate_source\": " << (p.source_inter >= 0 ? "true" : "false")
		  << ", \"result\": " << (p.id == plan.result_pipe ? "true" : "false") << "}";
	}
	o << "]";
	return o.str();
}

int vc_plan_describe(vc_engine* eng, const char* plan, const char* flavor, char* buf, size_t cap, size_t* len)
{
	return guarded([&] {
		if (!eng || !plan) {
			throw Error(VC_ERR_INVALID, "null argument");
		}
		const Flavor fl = Flavor::parse(flavor ? flavor : "");
		std::lock_guard<std::mutex> g(eng->e.mu);
		LoweredPlan lp = lower_plan(parse_plan(plan), eng->e.tables, fl, eng->e.dict);
		copy_out("{\"pipelines\": " + describe_pipelines(lp) + "}", buf, cap, len);
	});
}

int vc_query_info(vc_query* q, char* buf, size_t cap, size_t* len)
{
	return guarded([&] {
		if (!q) {
			throw Error(VC_ERR_INVALID, "null query");
		}
		Query& qq = q->q;
		std::ostringstream o;
		o << "{\"flavor\": \"" << qq.flavor.str() << "\", \"result_cols\": " << qq.plan.result_cols
		  << ", \"source_bytes\": " << qq.code.source.size() << ", \"pipelines\": " << describe_pipelines(qq.plan);
		o << ", \"kernels\": [";
		for (size_t i = 0; i < qq.code.launches.size(); i++) {
			auto& l = qq.code.launches[i];
			o << (i ? ", " : "") << "{\"name\": \"" << l.kernel << "\", \"pipeline\": " << l.pipe << ", \"smem\": "
			  << l.smem << ", \"threads\": " << l.threads << ", \"dominant\": " << (l.dominant ? "true" : "false") << "}";
		}
		o << "]}";
		copy_out(o.str(), buf, cap, len);
	});
}

int vc_query_source(vc_query* q, char* buf, size_t cap, size_t* len)
{
	return guarded([&] {
		if (!q) {
			throw Error(VC_ERR_INVALID, "null query");
		}
		copy_out(q->q.code.source, buf, cap, len);
	});
}

int vc_query_time(vc_query* q, int reps, int flush_l2, void* stream, float* ms_out, int cap)
{
	return guarded([&] {
		if (!q || reps < 1 || !ms_out || cap < reps) {
			throw Error(VC_ERR_INVALID, "bad arguments");
		}
		Query& qq = q->q;
		if (qq.eng->offline) {
			throw Error(VC_ERR_NO_DEVICE, "an offline engine only generates and compiles code");
		}
		VC_CHECK_CUDA(cudaSetDevice(qq.eng->device));
		cudaStream_t s = (cudaStream_t)stream;
		static thread_local void* flush = nullptr;
		static thread_local int flush_dev = -1;
		const size_t flush_bytes = 256ull << 20; /* larger than the 126 MiB L2 */
		if (flush_l2 && (flush == nullptr || flush_dev != qq.eng->device)) {
			VC_CHECK_CUDA(cudaMalloc(&flush, flush_bytes));
			flush_dev = qq.eng->device;
		}
		cudaEvent_t a, b;
		VC_CHECK_CUDA(cudaEventCreate(&a));
		VC_CHECK_CUDA(cudaEventCreate(&b));
		for (int r = 0; r < reps; r++) {
			if (flush_l2) {
				VC_CHECK_CUDA(cudaMemsetAsync(flush, r & 0xff, flush_bytes, s));
			}
			VC_CHECK_CUDA(cudaEventRecord(a, s));
			query_launch(qq, s);
			VC_CHECK_CUDA(cudaEventRecord(b, s));
			VC_CHECK_CUDA(cudaEventSynchronize(b));
			VC_CHECK_CUDA(cudaEventElapsedTime(&ms_out[r], a, b));
		}
		cudaEventDestroy(a);
		cudaEventDestroy(b);
		query_fetch(qq); /* surfaces device errors of the timed runs */
	});
}

int vc_query_profile(vc_query* q, int enable)
{
	return guarded([&] {
		if (!q) {
			throw Error(VC_ERR_INVALID, "null query");
		}
		q->q.profile = enable != 0;
	});
}

int vc_query_timings(vc_query* q, float* ms, int cap, int* n, char* names, size_t names_cap)
{
	return guarded([&] {
		if (!q) {
			throw Error(VC_ERR_INVALID, "null query");
		}
		query_fetch(q->q);
		const auto& t = q->q.last_ms;
		if (n) {
			*n = (int)t.size();
		}
		for (int i = 0; i < (int)t.size() && i < cap && ms; i++) {
			ms[i] = t[i];
		}
		std::string s;
		for (auto& l : q->q.code.launches) {
			s += l.kernel + "\n";
		}
		copy_out(s, names, names_cap, nullptr);
	});
}

} // extern "C"
