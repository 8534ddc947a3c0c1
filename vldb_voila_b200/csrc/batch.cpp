/*
 * Batched execution: many queries (pipelines of uneven sizes) in one persistent kernel.
 *
 * The reference runs one query at a time and, inside it, one pipeline at a time with
 * tbb::parallel_for over threads (runtime_framework.cpp:166-198).  Small pipelines leave
 * most of a GPU idle and every launch costs microseconds, so a batch instead fuses all
 * pipelines of all its queries into one launch: a persistent grid (one wave of CTAs) pulls
 * work items -- state clears, tile ranges of pipelines, slot ranges of group extraction --
 * from a device work queue in dependency order (see generate_batch).  The launch (clears
 * included) is captured once into a CUDA graph and replayed.
 *
 * Waits on dependencies are bounded (2 s unless vc_batch_set_wait_limit says otherwise); a
 * wait that gives up records VD_ERR_WAIT_TIMEOUT in the batch's error word and the item is
 * skipped (it still counts as done, so nothing waits on it in turn), so a stuck batch ends
 * with an error instead of a hang.
 */
#include <algorithm>
#include <cstring>
#include <functional>
#include <sstream>

#include "engine_internal.hpp"
#include "../../include/voila_cuda.h"

struct vc_query;

namespace vc {

int abi_guard_mlp(const std::function<void()>& f);
void query_mark_external_run(Query& q, cudaStream_t s);
void query_launch(Query& q, cudaStream_t stream);
Query* vc_query_internal(vc_query* q);

Batch::~Batch()
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
	for (void* p : allocations) {
		cudaFree(p);
	}
}

static void* balloc(Batch& b, size_t bytes)
{
	void* p = nullptr;
	VC_CHECK_CUDA(cudaMalloc(&p, std::max<size_t>(bytes, 256)));
	b.allocations.push_back(p);
	return p;
}

/* Clear items: every query's per-run state, in chunks of at most 8 MiB, placed just before
 * the query's first work item, with a done-counter per query that the query's first-phase
 * items wait for (a table cleared right before its pipeline runs can still be in L2 when the
 * pipeline reaches it).  Every dependency then points at items earlier in the queue, which is
 * what lets the persistent kernel's CTAs claim items in order without deadlock. */
static void add_clears_in_order(Batch& b, BatchCode& bc)
{
	const size_t nq = b.queries.size();
	std::vector<std::vector<BatchItem>> clears(nq);
	const int64_t chunk = 8ll << 20;
	for (size_t qi = 0; qi < nq; qi++) {
		QueryState& qst = state_of(*b.queries[qi]);
		std::vector<std::pair<void*, size_t>> all = qst.memsets;
		all.insert(all.end(), qst.clean_memsets.begin(), qst.clean_memsets.end());
		for (auto& m : all) {
			const int64_t bytes = (int64_t)((m.second + 15) & ~(size_t)15); /* allocations are 256-byte granular */
			const int64_t poff = (int64_t)bc.params.size();
			bc.params.push_back((unsigned long long)(uintptr_t)m.first);
			for (int64_t off = 0; off < bytes; off += chunk) {
				BatchItem it;
				it.shape = -1;
				it.dep = -1;
				it.params = poff;
				it.begin = off;
				it.end = std::min(off + chunk, bytes);
				it.nitems = 1;
				it.dep_target = 0;
				it.done = bc.ncounters + (int)qi;
				it.finish = -1;
				clears[qi].push_back(it);
			}
		}
	}
	auto query_of = [&](const BatchItem& it) {
		const auto& qb = bc.query_params_begin;
		return (size_t)(std::upper_bound(qb.begin(), qb.end(), it.params) - qb.begin()) - 1;
	};
	std::vector<BatchItem> ordered;
	ordered.reserve(bc.items.size() + 64);
	std::vector<bool> placed(nq, false);
	for (auto it : bc.items) {
		const size_t qi = query_of(it);
		if (qi >= nq) {
			throw Error(VC_ERR_INVALID, "batch item outside every query's parameters");
		}
		if (!placed[qi]) {
			ordered.insert(ordered.end(), clears[qi].begin(), clears[qi].end());
			placed[qi] = true;
		}
		if (it.dep_target == -2) {
			it.dep = bc.ncounters + (int)qi;
			it.dep_target = (int64_t)clears[qi].size();
		}
		ordered.push_back(it);
	}
	for (size_t qi = 0; qi < nq; qi++) {
		if (!placed[qi]) {
			ordered.insert(ordered.end(), clears[qi].begin(), clears[qi].end());
		}
	}
	bc.items.swap(ordered);
	bc.ncounters += (int)nq;
}

static void batch_prepare(Batch& b, const std::vector<Flavor>& flavors, int64_t tiles_per_item)
{
	/* a query prepared with a partitioned group-by runs it through a global group table here */
	for (Query* q : b.queries) {
		QueryState& st = state_of(*q);
		for (auto& p : q->plan.pipes) {
			if (p.sink.kind == Sink::AggHash && !st.pipes[p.id].sink_dev) {
				alloc_group_table(*q, p, st.pipes[p.id]);
			}
		}
	}
	if (b.eng->offline) {
		/* compile-only engines: generate and compile the batch module and build its work
		 * queue (on the host only, for inspection) */
		BatchCode bc = generate_batch(b.queries, flavors, b.flavor.threads, tiles_per_item);
		add_clears_in_order(b, bc);
		b.host_items = bc.items;
		b.source = bc.source;
		b.nitems = (int64_t)bc.items.size();
		b.smem = bc.smem;
		std::string log;
		jit_cubin(bc.source, &log);
		return;
	}
	VC_CHECK_CUDA(cudaSetDevice(b.eng->device));
	BatchCode bc = generate_batch(b.queries, flavors, b.flavor.threads, tiles_per_item);
	add_clears_in_order(b, bc);
	b.host_items = bc.items;
	b.nitems = (int64_t)bc.items.size();
	b.source = bc.source;
	std::string log;
	b.mod = jit_compile(bc.source, &log);
	VC_CHECK_CUDA(cudaLibraryGetKernel(&b.kernel, b.mod->lib, "vc_batch"));
	b.smem = bc.smem;
	cudaFuncAttributes fa;
	VC_CHECK_CUDA(cudaFuncGetAttributes(&fa, (const void*)b.kernel));
	b.regs = fa.numRegs;
	if (b.smem > 0) {
		/* batches of one shape share the kernel: the limit only grows */
		if ((size_t)fa.maxDynamicSharedSizeBytes < b.smem) {
			VC_CHECK_CUDA(cudaFuncSetAttribute((const void*)b.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
				(int)b.smem));
		}
	}
	VC_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b.occupancy, (const void*)b.kernel, b.flavor.threads,
		b.smem));
	if (b.occupancy < 1) {
		throw Error(VC_ERR_UNSUPPORTED, "the batch kernel cannot be resident with its shared memory");
	}
	/* one wave only: every CTA is resident, so a CTA waiting on a dependency never waits
	 * for a CTA that cannot run */
	b.grid = b.eng->sms * b.occupancy;

	b.items = (BatchItem*)balloc(b, sizeof(BatchItem) * bc.items.size());
	VC_CHECK_CUDA(cudaMemcpy(b.items, bc.items.data(), sizeof(BatchItem) * bc.items.size(), cudaMemcpyHostToDevice));
	b.params = (unsigned long long*)balloc(b, sizeof(unsigned long long) * std::max<size_t>(bc.params.size(), 1));
	VC_CHECK_CUDA(cudaMemcpy(b.params, bc.params.data(), sizeof(unsigned long long) * bc.params.size(),
		cudaMemcpyHostToDevice));
	b.counters_bytes = sizeof(unsigned long long) * (size_t)bc.ncounters;
	b.counters = (unsigned long long*)balloc(b, b.counters_bytes + sizeof(unsigned long long) * (b.queries.size() + 1) + 64);
	b.finish = b.counters + bc.ncounters;
	b.err = (unsigned*)(b.finish + b.queries.size() + 1);
}

static void batch_launch_all(Batch& b, cudaStream_t s)
{
	const size_t book = b.counters_bytes + sizeof(unsigned long long) * (b.queries.size() + 1) + 64;
	VC_CHECK_CUDA(cudaMemsetAsync(b.counters, 0, book, s));
	long long nwork = b.nitems;
	int nq = (int)b.queries.size();
	void* args[] = {&b.items, &nwork, &b.counters, &b.params, &b.finish, &nq, &b.err, &b.wait_ns};
	VC_CHECK_CUDA(cudaLaunchKernel((const void*)b.kernel, dim3((unsigned)b.grid), dim3((unsigned)b.flavor.threads), args,
		b.smem, s));
}

static void batch_run(Batch& b, cudaStream_t s)
{
	VC_CHECK_CUDA(cudaSetDevice(b.eng->device));
	if (!b.graph) {
		cudaStream_t cs;
		VC_CHECK_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
		cudaGraph_t g;
		VC_CHECK_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
		try {
			batch_launch_all(b, cs);
		} catch (...) {
			cudaStreamEndCapture(cs, &g);
			cudaStreamDestroy(cs);
			throw;
		}
		VC_CHECK_CUDA(cudaStreamEndCapture(cs, &g));
		VC_CHECK_CUDA(cudaGraphInstantiate(&b.graph, g, 0));
		cudaGraphDestroy(g);
		cudaStreamDestroy(cs);
	}
	VC_CHECK_CUDA(cudaGraphLaunch(b.graph, s));
	b.stream = s;
	for (Query* q : b.queries) {
		query_mark_external_run(*q, s);
	}
}

} // namespace vc

using namespace vc;

/* A batch: the queries that run in the persistent kernel (b), and those whose largest
 * pipeline has at least solo_rows rows, which run as their own launches (each with its own
 * flavor's kernels: the persistent kernel's lean shapes would only slow a pipeline that fills
 * the GPU by itself) on the same stream after it. */
struct vc_batch {
	Batch b;
	bool has_batch = false;
	std::vector<Query*> solo;
	std::vector<int> slot;          /* per query: its index in b.queries, or -(solo index + 1) */
	cudaEvent_t ev0 = nullptr;      /* before the batch's first launch */
	std::vector<cudaEvent_t> ev;    /* after each solo query */
	cudaStream_t stream = nullptr;  /* the stream of the last run */
	bool offline = false;
	~vc_batch()
	{
		if (offline) {
			return;
		}
		if (ev0) {
			cudaEventDestroy(ev0);
		}
		for (auto e : ev) {
			cudaEventDestroy(e);
		}
	}
};

extern "C" {

static int64_t query_rows(const Query& q)
{
	int64_t r = 0;
	for (const auto& p : q.plan.pipes) {
		r = std::max(r, p.rows);
	}
	return r;
}

int vc_batch_new_split(vc_query** queries, int n, const char** flavors, int threads, int64_t tiles_per_item,
	int64_t solo_rows, vc_batch** out)
{
	vc_batch* h = nullptr;
	int rc = abi_guard_mlp([&] {
		if (!queries || n < 1 || !out || threads < 32 || threads > 1024 || threads % 32 || tiles_per_item < 1 ||
			solo_rows < 0) {
			throw Error(VC_ERR_INVALID, "bad batch arguments");
		}
		h = new vc_batch();
		std::vector<Flavor> fls;
		Engine* eng = nullptr;
		for (int i = 0; i < n; i++) {
			if (!queries[i]) {
				throw Error(VC_ERR_INVALID, "null query in batch");
			}
			Query* q = vc_query_internal(queries[i]);
			if (eng && eng->device != q->eng->device) {
				throw Error(VC_ERR_INVALID, "batched queries must live on one device");
			}
			if (eng && eng->offline != q->eng->offline) {
				throw Error(VC_ERR_INVALID, "a batch cannot mix offline and device queries");
			}
			eng = q->eng;
			if (solo_rows > 0 && query_rows(*q) >= solo_rows) {
				h->slot.push_back(-(int)h->solo.size() - 1);
				h->solo.push_back(q);
				continue;
			}
			h->slot.push_back((int)h->b.queries.size());
			h->b.queries.push_back(q);
			fls.push_back(flavors && flavors[i] ? Flavor::parse(flavors[i]) : q->flavor);
		}
		h->b.eng = eng;
		h->offline = eng->offline;
		h->b.flavor.threads = threads;
		h->has_batch = !h->b.queries.empty();
		if (h->has_batch) {
			batch_prepare(h->b, fls, tiles_per_item);
		}
		*out = h;
	});
	if (rc != VC_OK && h) {
		delete h; /* the error message of the failed call stays in place */
	}
	return rc;
}

int vc_batch_new(vc_query** queries, int n, const char** flavors, int threads, int64_t tiles_per_item, vc_batch** out)
{
	return vc_batch_new_split(queries, n, flavors, threads, tiles_per_item, 0, out);
}

int vc_batch_run(vc_batch* h, void* stream)
{
	return abi_guard_mlp([&] {
		if (!h) {
			throw Error(VC_ERR_INVALID, "null batch");
		}
		if (h->b.eng->offline) {
			throw Error(VC_ERR_NO_DEVICE, "an offline engine only generates and compiles code");
		}
		VC_CHECK_CUDA(cudaSetDevice(h->b.eng->device));
		h->stream = (cudaStream_t)stream;
		if (!h->solo.empty()) {
			if (!h->ev0) {
				VC_CHECK_CUDA(cudaEventCreate(&h->ev0));
				h->ev.assign(h->solo.size(), nullptr);
				for (auto& e : h->ev) {
					VC_CHECK_CUDA(cudaEventCreate(&e));
				}
			}
			VC_CHECK_CUDA(cudaEventRecord(h->ev0, h->stream));
		}
		if (h->has_batch) {
			batch_run(h->b, h->stream);
		}
		for (size_t k = 0; k < h->solo.size(); k++) {
			query_launch(*h->solo[k], h->stream);
			VC_CHECK_CUDA(cudaEventRecord(h->ev[k], h->stream));
		}
	});
}

int vc_batch_wait(vc_batch* h)
{
	return abi_guard_mlp([&] {
		if (!h) {
			throw Error(VC_ERR_INVALID, "null batch");
		}
		Batch& b = h->b;
		VC_CHECK_CUDA(cudaSetDevice(b.eng->device));
		VC_CHECK_CUDA(cudaStreamSynchronize(h->stream));
		if (!h->has_batch) {
			return;
		}
		unsigned err = 0;
		VC_CHECK_CUDA(cudaMemcpy(&err, b.err, sizeof(err), cudaMemcpyDeviceToHost));
		if (err) {
			/* skipped items may leave the queries' self-cleaning tables set */
			for (Query* q : b.queries) {
				q->dirty = true;
			}
		}
		if (err & 2u) {
			throw Error(VC_ERR_TIMEOUT, "a batch dependency wait gave up");
		}
		if (err) {
			throw Error(VC_ERR_CAPACITY, "batch error bits " + std::to_string(err));
		}
	});
}

int vc_batch_latencies(vc_batch* h, double* us, int n)
{
	return abi_guard_mlp([&] {
		if (!h || !us || n < (int)h->slot.size()) {
			throw Error(VC_ERR_INVALID, "bad arguments");
		}
		Batch& b = h->b;
		VC_CHECK_CUDA(cudaSetDevice(b.eng->device));
		VC_CHECK_CUDA(cudaStreamSynchronize(h->stream));
		std::vector<unsigned long long> f(b.queries.size() + 1, 0ull);
		if (h->has_batch) {
			VC_CHECK_CUDA(cudaMemcpy(f.data(), b.finish, sizeof(unsigned long long) * f.size(), cudaMemcpyDeviceToHost));
		}
		const unsigned long long start = f.back();
		for (size_t i = 0; i < h->slot.size(); i++) {
			const int k = h->slot[i];
			if (k >= 0) {
				/* the persistent kernel's clock from its start */
				us[i] = f[(size_t)k] >= start ? (double)(f[(size_t)k] - start) / 1000.0 : -1.0;
			} else {
				/* events from the batch's first launch to the solo query's end */
				float ms = -1.0f;
				if (h->ev0 && cudaEventElapsedTime(&ms, h->ev0, h->ev[(size_t)(-k - 1)]) != cudaSuccess) {
					ms = -1.0f;
				}
				us[i] = ms >= 0.0f ? (double)ms * 1000.0 : -1.0;
			}
		}
	});
}

int vc_batch_info(vc_batch* h, char* buf, size_t cap, size_t* len)
{
	return abi_guard_mlp([&] {
		if (!h) {
			throw Error(VC_ERR_INVALID, "null batch");
		}
		Batch& b = h->b;
		std::ostringstream o;
		o << "{\"queries\": " << h->slot.size() << ", \"batched\": " << b.queries.size() << ", \"solo\": "
		  << h->solo.size() << ", \"work_items\": " << b.nitems << ", \"grid\": " << b.grid
		  << ", \"threads\": " << b.flavor.threads << ", \"smem\": " << b.smem << ", \"regs\": " << b.regs
		  << ", \"occupancy\": " << b.occupancy
		  << ", \"source_bytes\": " << b.source.size() << "}";
		const std::string s = o.str();
		if (len) {
			*len = s.size();
		}
		if (buf && cap) {
			const size_t k = std::min(cap - 1, s.size());
			std::memcpy(buf, s.data(), k);
			buf[k] = 0;
		}
	});
}

int vc_batch_source(vc_batch* h, char* buf, size_t cap, size_t* len)
{
	return abi_guard_mlp([&] {
		if (!h) {
			throw Error(VC_ERR_INVALID, "null batch");
		}
		const std::string& s = h->b.source;
		if (len) {
			*len = s.size();
		}
		if (buf && cap) {
			const size_t k = std::min(cap - 1, s.size());
			std::memcpy(buf, s.data(), k);
			buf[k] = 0;
		}
	});
}

int vc_batch_items(vc_batch* h, int64_t* out, int64_t cap, int64_t* n)
{
	return abi_guard_mlp([&] {
		if (!h) {
			throw Error(VC_ERR_INVALID, "null batch");
		}
		const auto& items = h->b.host_items;
		if (n) {
			*n = (int64_t)items.size();
		}
		if (!out) {
			return;
		}
		const int64_t k = std::min<int64_t>(cap, (int64_t)items.size());
		for (int64_t i = 0; i < k; i++) {
			const BatchItem& it = items[(size_t)i];
			int64_t* r = out + 8 * i;
			r[0] = it.shape;
			r[1] = it.dep;
			r[2] = it.dep_target;
			r[3] = it.done;
			r[4] = it.nitems;
			r[5] = it.begin;
			r[6] = it.end;
			r[7] = it.params;
		}
	});
}

int vc_batch_set_wait_limit(vc_batch* h, uint64_t ns)
{
	return abi_guard_mlp([&] {
		if (!h || ns < 1000 || ns > 60000000000ull) {
			throw Error(VC_ERR_INVALID, "wait limit must be between 1 us and 60 s");
		}
		Batch& b = h->b;
		if (b.wait_ns != ns) {
			b.wait_ns = ns;
			if (b.graph) {
				/* the limit is a kernel argument of the captured launch */
				VC_CHECK_CUDA(cudaGraphExecDestroy(b.graph));
				b.graph = nullptr;
			}
		}
	});
}

int vc_batch_hold_item(vc_batch* h, int64_t index, int hold)
{
	return abi_guard_mlp([&] {
		if (!h || index < 0 || index >= h->b.nitems) {
			throw Error(VC_ERR_INVALID, "no such work item");
		}
		Batch& b = h->b;
		if (b.eng->offline) {
			throw Error(VC_ERR_NO_DEVICE, "an offline engine only generates and compiles code");
		}
		VC_CHECK_CUDA(cudaSetDevice(b.eng->device));
		if (b.stream) {
			VC_CHECK_CUDA(cudaStreamSynchronize(b.stream));
		}
		auto it = std::find(b.held_index.begin(), b.held_index.end(), index);
		BatchItem item = b.host_items[(size_t)index];
		if (hold) {
			if (it == b.held_index.end()) {
				b.held_index.push_back(index);
				b.held.push_back(item);
			}
			/* the clears' counter never reaches this: the item's bounded wait runs out */
			item.dep = 1;
			item.dep_target = (int64_t)1 << 62;
		} else {
			if (it == b.held_index.end()) {
				return;
			}
			const size_t k = (size_t)(it - b.held_index.begin());
			item = b.held[k];
			b.held.erase(b.held.begin() + (long)k);
			b.held_index.erase(it);
		}
		b.host_items[(size_t)index] = item;
		VC_CHECK_CUDA(cudaMemcpy(b.items + index, &item, sizeof(BatchItem), cudaMemcpyHostToDevice));
	});
}

int vc_batch_free(vc_batch* h)
{
	return abi_guard_mlp([&] { delete h; });
}

} // extern "C"
