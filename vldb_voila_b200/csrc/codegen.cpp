/*
 * CUDA code generator: one fused kernel per lowered pipeline.
 *
 * This is the CUDA counterpart of the reference's per-pipeline code generators
 * (cg_hyper.cpp gen_pipeline :804-845, cg_vector.cpp :793-923): where those emit a
 * tuple-at-a-time loop or a chain of vector primitives, this emits a CUDA kernel in which
 * every thread owns `rows` consecutive rows of a tile (vector loads), evaluates the
 * pipeline's filters and probes for all of them (op-major, so independent hash-table loads
 * overlap) and feeds its sink.  Per pipeline sink:
 *
 *   JoinBuild  materialise  (compacted packed keys/payloads/hashes; write/write_pos,
 *                            relalg_translator.cpp:828-907)
 *              clear + insert (bucket_build; runtime_struct.cpp:1283-1324)
 *   AggGlobal  registers -> block reduction -> one atomic per CTA (aggr_gsum/gcount)
 *   AggDense   shared-memory slots over the key domain, warp-combined updates, merged
 *              into a global slot array at CTA end; extract kernel emits count > 0 slots
 *   AggHash    global open-addressing group table, warp-combined leader updates,
 *              optional per-CTA shared-memory cache for hot keys; extract kernel
 *   Emit       warp-aggregated append of the selected rows
 *
 * The source depends only on the plan's shape (column types, operators, aggregate count)
 * and the flavor knobs.  Every data-dependent number (row counts, constants, key ranges,
 * pointers) is a kernel parameter, so one compiled module serves every instance of a shape.
 */
#include <algorithm>
#include <sstream>

#include "engine_internal.hpp"

namespace vc {

static const char* ctype(int t)
{
	switch (t) {
	case VC_TYPE_U8: return "uint8_t";
	case VC_TYPE_I16: return "int16_t";
	case VC_TYPE_I32: return "int32_t";
	default: return "int64_t";
	}
}

static int64_t pow2_at_least(int64_t x)
{
	int64_t p = 1;
	while (p < x) {
		p <<= 1;
	}
	return p;
}

namespace {

struct PipeGen {
	Pipeline& p;
	LoweredPlan& plan;
	const Flavor& fl;
	std::vector<unsigned long long>& params;
	std::ostringstream o;
	std::string name;
	int V;

	PipeGen(Pipeline& pp, LoweredPlan& pl, const Flavor& f, std::vector<unsigned long long>& prm)
		: p(pp), plan(pl), fl(f), params(prm), V(f.rows) {
		name = "vc_p" + std::to_string(p.id);
	}

	/* allocates a parameter slot holding `v`; returns its C expression */
	std::string P(unsigned long long v) {
		params.push_back(v);
		return "((int64_t)p.v[" + std::to_string(params.size() - 1) + "])";
	}
	std::string Pu(unsigned long long v) {
		params.push_back(v);
		return "((uint64_t)p.v[" + std::to_string(params.size() - 1) + "])";
	}
	std::string Pptr(const void* ptr, const std::string& type) {
		params.push_back((unsigned long long)(uintptr_t)ptr);
		return "((" + type + ")p.v[" + std::to_string(params.size() - 1) + "])";
	}

	/* C expression for e at row index `v` */
	std::string expr(const BExprP& e, const std::string& v) {
		switch (e->kind) {
		case BExpr::Col:
			return "((int64_t)x" + std::to_string(e->col) + "[" + v + "])";
		case BExpr::Const:
			if (e->param < 0) {
				params.push_back((unsigned long long)e->cval);
				e->param = (int)params.size() - 1;
			}
			return "((int64_t)p.v[" + std::to_string(e->param) + "])";
		case BExpr::ProbeOut:
			return "pay" + std::to_string(e->probe) + "_" + std::to_string(e->pidx) + "[" + v + "]";
		case BExpr::Fun: {
			static const std::map<std::string, std::string> ops = {
				{"add", "+"}, {"sub", "-"}, {"mul", "*"}, {"lt", "<"}, {"le", "<="}, {"gt", ">"},
				{"ge", ">="}, {"eq", "=="}, {"ne", "!="}, {"and", "&&"}, {"or", "||"}};
			return "(" + expr(e->args[0], v) + " " + ops.at(e->fn) + " " + expr(e->args[1], v) + ")";
		}
		}
		return "0";
	}

	int A() const { return (int)p.sink.aggs.size(); }

	std::string agg_vals(const std::string& v) {
		std::ostringstream s;
		s << "int64_t vals[" << A() << "] = {";
		for (int a = 0; a < A(); a++) {
			const auto& ag = p.sink.aggs[a];
			s << (a ? ", " : "") << (ag.count ? std::string("(int64_t)1") : expr(ag.arg, v));
		}
		s << "};";
		return s.str();
	}

	/* hash of the raw key values, as the reference's hash/rehash chain computes it */
	std::string key_hash(const std::vector<BExprP>& keys, const std::string& v) {
		std::string h = "vd::hash(" + expr(keys[0], v) + ")";
		for (size_t i = 1; i < keys.size(); i++) {
			h = "vd::rehash(" + h + ", " + expr(keys[i], v) + ")";
		}
		return h;
	}

	void header(const std::string& kname, int threads) {
		o << "extern \"C\" __global__ void __launch_bounds__(" << threads << ") " << kname
		  << "(const VcParams p) {\n";
	}

	/* ------------------------------------------------------------ main kernel ------ */

	std::string gen_main(size_t& smem_out) {
		std::ostringstream body;
		const int T = fl.threads;
		smem_out = 0;

		header(name + "_main", T);
		o << "  const int64_t n = " << P((unsigned long long)p.rows) << ";\n";
		p.err_slot = (int)params.size();
		err_slot = params.size();
		o << "  unsigned* const err = (unsigned*)p.v[" << params.size() << "];\n";
		params.push_back(0); /* error word, filled by the runtime */
		p.col_slots.clear();
		for (size_t c = 0; c < p.cols.size(); c++) {
			p.col_slots.push_back((int)params.size());
			o << "  const " << ctype(p.cols[c].type) << "* __restrict__ c" << c << " = (const "
			  << ctype(p.cols[c].type) << "*)p.v[" << params.size() << "];\n";
			params.push_back(0); /* column pointer, filled by the runtime */
		}
		o << "  (void)err;\n";

		sink_prologue(smem_out);

		o << "  const int64_t tile = (int64_t)" << T << " * " << V << ";\n";
		o << "  const int64_t ntiles = (n + tile - 1) / tile;\n";
		o << "  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {\n";
		o << "    const int64_t r0 = t * tile + (int64_t)threadIdx.x * " << V << ";\n";
		o << "    bool act[" << V << "];\n";
		o << "#pragma unroll\n    for (int v = 0; v < " << V << "; v++) { act[v] = r0 + v < n; }\n";
		for (size_t c = 0; c < p.cols.size(); c++) {
			o << "    " << ctype(p.cols[c].type) << " x" << c << "[" << V << "];\n";
			o << "    vd::load_rows<" << ctype(p.cols[c].type) << ", " << V << ">(c" << c << ", r0, n, x" << c << ");\n";
		}
		/* ops, op-major */
		for (size_t i = 0; i < p.ops.size(); i++) {
			const Op& op = p.ops[i];
			if (op.kind == Op::Filter) {
				o << "#pragma unroll\n    for (int v = 0; v < " << V << "; v++) { act[v] = act[v] && "
				  << expr(op.pred, "v") << "; }\n";
			} else {
				gen_probe((int)i, op);
			}
		}
		sink_row();
		o << "  }\n";
		sink_epilogue();
		o << "}\n\n";
		return o.str();
	}

	void gen_probe(int opi, const Op& op) {
		JoinDesc& jd = plan.joins[op.join];
		if (!jd.join01) {
			throw Error(6, "joinN probes are not supported by the CUDA flavor yet");
		}
		const std::string KT = jd.key64 ? "uint64_t" : "uint32_t";
		const std::string PT = jd.pay64 ? "uint64_t" : "uint32_t";
		const std::string S = "vd::JoinSlot<" + KT + ", " + PT + ">";
		const std::string j = std::to_string(opi);
		for (int k = 0; k < op.npay; k++) {
			o << "    int64_t pay" << j << "_" << k << "[" << V << "];\n";
		}
		o << "    {\n";
		o << "      const " << S << "* __restrict__ jt = " << Pptr(jd.table, "const " + S + "*") << ";\n";
		o << "      const uint64_t bmask = ((const unsigned long long*)" << Pptr(jd.words, "const void*")
		  << ")[1];\n";
		o << "      int st[" << V << "]; uint64_t bk[" << V << "]; " << KT << " key[" << V << "]; " << PT
		  << " raw[" << V << "];\n";
		o << "#pragma unroll\n      for (int v = 0; v < " << V << "; v++) {\n";
		std::string inrange = "act[v]";
		std::string packed = "0ull";
		for (size_t k = 0; k < op.keys.size(); k++) {
			const std::string kv = expr(op.keys[k], "v");
			const std::string lo = P((unsigned long long)(int64_t)jd.key_b[k].lo);
			const std::string hi = P((unsigned long long)(int64_t)jd.key_b[k].hi);
			inrange += " && " + kv + " >= " + lo + " && " + kv + " <= " + hi;
			packed += " | ((uint64_t)(" + kv + " - " + lo + ") << " + P((unsigned long long)jd.key_shift[k]) + ")";
		}
		o << "        const bool ok = " << inrange << ";\n";
		o << "        key[v] = (" << KT << ")((" << packed << ") + 1ull);\n";
		o << "        bk[v] = " << key_hash(op.keys, "v") << " & bmask;\n";
		o << "        raw[v] = 0; st[v] = 0;\n";
		o << "        if (ok) { st[v] = vd::join_probe_bucket(jt, bk[v], key[v], raw[v]); }\n";
		o << "      }\n";
		o << "#pragma unroll\n      for (int v = 0; v < " << V << "; v++) {\n";
		o << "        int guard = 0;\n";
		o << "        while (st[v] == 2) {\n";
		o << "          if (++guard > VD_MAX_PROBES) { atomicOr(err, VD_ERR_TABLE_FULL); st[v] = 0; break; }\n";
		o << "          bk[v] = (bk[v] + 1) & bmask;\n";
		o << "          st[v] = vd::join_probe_bucket(jt, bk[v], key[v], raw[v]);\n";
		o << "        }\n";
		o << "        act[v] = st[v] == 1;\n";
		for (int k = 0; k < op.npay; k++) {
			const int bits = (k + 1 < op.npay ? jd.pay_shift[k + 1] : jd.pay_bits) - jd.pay_shift[k];
			const unsigned long long mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1ull);
			o << "        pay" << j << "_" << k << "[v] = " << P((unsigned long long)(int64_t)jd.pay_b[k].lo)
			  << " + (int64_t)(((uint64_t)raw[v] >> " << P((unsigned long long)jd.pay_shift[k]) << ") & "
			  << Pu(mask) << ");\n";
		}
		o << "      }\n";
		o << "    }\n";
	}

	/* ------------------------------------------------------------ sinks ------------ */

	void sink_prologue(size_t& smem) {
		Sink& s = p.sink;
		switch (s.kind) {
		case Sink::AggGlobal:
			o << "  int64_t acc[" << A() << "];\n";
			o << "#pragma unroll\n  for (int a = 0; a < " << A() << "; a++) { acc[a] = 0; }\n";
			break;
		case Sink::AggDense: {
			const int64_t D = (int64_t)s.domain;
			const bool in_smem = D * A() * 8 <= 96 * 1024;
			if (in_smem) {
				smem = (size_t)(D * A() * 8);
				o << "  extern __shared__ __align__(16) unsigned char vd_smem[];\n";
				o << "  unsigned long long* const sacc = (unsigned long long*)vd_smem;\n";
				o << "  for (int64_t i = threadIdx.x; i < " << P((unsigned long long)(D * A()))
				  << "; i += blockDim.x) { sacc[i] = 0ull; }\n";
				o << "  __syncthreads();\n";
			} else {
				o << "  unsigned long long* const sacc = " << Pptr(s_dev(), "unsigned long long*") << ";\n";
			}
			dense_in_smem = in_smem;
			break;
		}
		case Sink::AggHash:
			o << "  unsigned long long* const gtab = " << Pptr(s_dev(), "unsigned long long*") << ";\n";
			o << "  const uint64_t gmask = " << Pu((unsigned long long)(s_cap() - 1)) << ";\n";
			if (fl.aggr == "cache") {
				const int S = (int)pow2_at_least(std::max(32, fl.cache_slots));
				smem = (size_t)S * (1 + A()) * 8;
				o << "  extern __shared__ __align__(16) unsigned char vd_smem[];\n";
				o << "  unsigned long long* const scache = (unsigned long long*)vd_smem;\n";
				o << "  for (int i = threadIdx.x; i < " << S * (1 + A()) << "; i += blockDim.x) { scache[i] = 0ull; }\n";
				o << "  __syncthreads();\n";
				cache_slots = S;
			}
			break;
		case Sink::JoinBuild: {
			JoinDesc& jd = plan.joins[s.join];
			o << "  unsigned long long* const words = " << Pptr(jd.words, "unsigned long long*") << ";\n";
			o << "  " << (jd.key64 ? "uint64_t" : "uint32_t") << "* const skeys = "
			  << Pptr(jd.stage_keys, jd.key64 ? "uint64_t*" : "uint32_t*") << ";\n";
			o << "  " << (jd.pay64 ? "uint64_t" : "uint32_t") << "* const spay = "
			  << Pptr(jd.stage_pay, jd.pay64 ? "uint64_t*" : "uint32_t*") << ";\n";
			o << "  uint64_t* const shash = " << Pptr(stage_hash(jd), "uint64_t*") << ";\n";
			break;
		}
		case Sink::Emit:
			o << "  int64_t* const out = " << Pptr(plan_out, "int64_t*") << ";\n";
			o << "  const int64_t ocap = " << P((unsigned long long)plan_out_cap) << ";\n";
			o << "  unsigned long long* const ocount = " << Pptr(out_count(), "unsigned long long*") << ";\n";
			break;
		}
	}

	void sink_row() {
		Sink& s = p.sink;
		switch (s.kind) {
		case Sink::AggGlobal:
			o << "#pragma unroll\n    for (int v = 0; v < " << V << "; v++) {\n";
			o << "      " << agg_vals("v") << "\n";
			o << "#pragma unroll\n      for (int a = 0; a < " << A() << "; a++) { acc[a] += act[v] ? vals[a] : 0; }\n";
			o << "    }\n";
			break;
		case Sink::AggDense: {
			o << "#pragma unroll\n    for (int v = 0; v < " << V << "; v++) {\n";
			std::string slot = "0";
			for (size_t k = 0; k < s.keys.size(); k++) {
				slot += " + (" + expr(s.keys[k], "v") + " - " + P((unsigned long long)(int64_t)s.keys[k]->b.lo) +
					") * " + P((unsigned long long)s.key_radix[k]);
			}
			o << "      const int64_t slot = act[v] ? (" << slot << ") : 0;\n";
			o << "      " << agg_vals("v") << "\n";
			o << "      if (vd::warp_combine<" << A() << ">((uint64_t)slot, act[v], vals)) {\n";
			o << "#pragma unroll\n        for (int a = 0; a < " << A() << "; a++) { atomicAdd(&sacc[slot * "
			  << A() << " + a], (unsigned long long)vals[a]); }\n";
			o << "      }\n    }\n";
			break;
		}
		case Sink::AggHash: {
			o << "#pragma unroll\n    for (int v = 0; v < " << V << "; v++) {\n";
			std::string packed = "0ull";
			for (size_t k = 0; k < s.keys.size(); k++) {
				packed += " | ((uint64_t)(" + expr(s.keys[k], "v") + " - " +
					P((unsigned long long)(int64_t)s.keys[k]->b.lo) + ") << " +
					P((unsigned long long)s.key_shift[k]) + ")";
			}
			o << "      const uint64_t pk = act[v] ? (" << packed << ") : 0ull;\n";
			o << "      " << agg_vals("v") << "\n";
			o << "      if (vd::warp_combine<" << A() << ">(pk, act[v], vals)) {\n";
			o << "        const uint64_t h = " << key_hash(s.keys, "v") << ";\n";
			if (fl.aggr == "cache") {
				o << "        if (!vd::cache_add<" << A() << ">(scache, " << cache_slots << ", h, pk + 1ull, vals)) {\n";
				o << "          vd::group_add<" << A() << ">(gtab, gmask, h, pk + 1ull, vals, err);\n";
				o << "        }\n";
			} else {
				o << "        vd::group_add<" << A() << ">(gtab, gmask, h, pk + 1ull, vals, err);\n";
			}
			o << "      }\n    }\n";
			break;
		}
		case Sink::JoinBuild: {
			JoinDesc& jd = plan.joins[s.join];
			o << "#pragma unroll\n    for (int v = 0; v < " << V << "; v++) {\n";
			o << "      const int64_t pos = vd::warp_append(&words[0], act[v]);\n";
			o << "      if (act[v]) {\n";
			std::string pk = "0ull";
			for (size_t k = 0; k < s.keys.size(); k++) {
				pk += " | ((uint64_t)(" + expr(s.keys[k], "v") + " - " + P((unsigned long long)(int64_t)jd.key_b[k].lo) +
					") << " + P((unsigned long long)jd.key_shift[k]) + ")";
			}
			std::string pp = "0ull";
			for (size_t k = 0; k < s.pay.size(); k++) {
				pp += " | ((uint64_t)(" + expr(s.pay[k], "v") + " - " + P((unsigned long long)(int64_t)jd.pay_b[k].lo) +
					") << " + P((unsigned long long)jd.pay_shift[k]) + ")";
			}
			o << "        skeys[pos] = (" << (jd.key64 ? "uint64_t" : "uint32_t") << ")((" << pk << ") + 1ull);\n";
			o << "        spay[pos] = (" << (jd.pay64 ? "uint64_t" : "uint32_t") << ")(" << pp << ");\n";
			o << "        shash[pos] = " << key_hash(s.keys, "v") << ";\n";
			o << "      }\n    }\n";
			break;
		}
		case Sink::Emit: {
			o << "#pragma unroll\n    for (int v = 0; v < " << V << "; v++) {\n";
			o << "      const int64_t pos = vd::warp_append(ocount, act[v]);\n";
			o << "      if (act[v]) {\n";
			o << "        if (pos < ocap) {\n";
			for (size_t c = 0; c < s.outs.size(); c++) {
				o << "          out[" << c << " * ocap + pos] = " << expr(s.outs[c], "v") << ";\n";
			}
			o << "        } else { atomicOr(err, VD_ERR_TABLE_FULL); }\n";
			o << "      }\n    }\n";
			break;
		}
		}
	}

	void sink_epilogue() {
		Sink& s = p.sink;
		switch (s.kind) {
		case Sink::AggGlobal:
			o << "  __shared__ int64_t red[32 * " << A() << "];\n";
			o << "  vd::block_sum<" << A() << ">(acc, red);\n";
			o << "  if (threadIdx.x == 0) {\n";
			o << "    unsigned long long* g = " << Pptr(s_dev(), "unsigned long long*") << ";\n";
			o << "#pragma unroll\n    for (int a = 0; a < " << A() << "; a++) { if (acc[a]) atomicAdd(&g[a], (unsigned long long)acc[a]); }\n";
			o << "  }\n";
			break;
		case Sink::AggDense:
			if (dense_in_smem) {
				const int64_t D = (int64_t)s.domain;
				o << "  __syncthreads();\n";
				o << "  {\n    unsigned long long* g = " << Pptr(s_dev(), "unsigned long long*") << ";\n";
				o << "    for (int64_t i = threadIdx.x; i < " << P((unsigned long long)D) << "; i += blockDim.x) {\n";
				o << "      if (sacc[i * " << A() << " + " << s.count_idx << "]) {\n";
				o << "#pragma unroll\n        for (int a = 0; a < " << A() << "; a++) { atomicAdd(&g[i * " << A()
				  << " + a], sacc[i * " << A() << " + a]); }\n";
				o << "      }\n    }\n  }\n";
			}
			break;
		case Sink::AggHash:
			if (fl.aggr == "cache") {
				o << "  __syncthreads();\n";
				o << "  for (int i = threadIdx.x; i < " << cache_slots << "; i += blockDim.x) {\n";
				o << "    const unsigned long long sk = scache[i * " << (1 + A()) << "];\n";
				o << "    if (sk != 0ull) {\n";
				o << "      int64_t vals[" << A() << "];\n";
				o << "#pragma unroll\n      for (int a = 0; a < " << A() << "; a++) { vals[a] = (int64_t)scache[i * "
				  << (1 + A()) << " + 1 + a]; }\n";
				/* recompute the hash of the raw key values from the packed key */
				o << "      const uint64_t pk = sk - 1ull;\n";
				std::string h;
				for (size_t k = 0; k < s.keys.size(); k++) {
					const int bits = (k + 1 < s.keys.size() ? s.key_shift[k + 1] : s.key_bits) - s.key_shift[k];
					const unsigned long long mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1ull);
					const std::string kv = "(" + P((unsigned long long)(int64_t)s.keys[k]->b.lo) + " + (int64_t)((pk >> " +
						P((unsigned long long)s.key_shift[k]) + ") & " + Pu(mask) + "))";
					h = k == 0 ? "vd::hash(" + kv + ")" : "vd::rehash(" + h + ", " + kv + ")";
				}
				o << "      vd::group_add<" << A() << ">(gtab, gmask, " << h << ", sk, vals, err);\n";
				o << "    }\n  }\n";
			}
			break;
		default:
			break;
		}
	}

	/* ------------------------------------------------------------ extra kernels ---- */

	/* join build: clear the table for the materialised count, then insert */
	std::string gen_join_build() {
		JoinDesc& jd = plan.joins[p.sink.join];
		const std::string KT = jd.key64 ? "uint64_t" : "uint32_t";
		const std::string PT = jd.pay64 ? "uint64_t" : "uint32_t";
		const std::string S = "vd::JoinSlot<" + KT + ", " + PT + ">";
		std::ostringstream k;
		const std::string words = Pptr(jd.words, "unsigned long long*");
		const std::string table = Pptr(jd.table, S + "*");
		k << "extern \"C\" __global__ void __launch_bounds__(256) " << name << "_clear(const VcParams p) {\n";
		k << "  unsigned long long* const words = " << words << ";\n";
		k << "  " << S << "* const jt = " << table << ";\n";
		k << "  const uint64_t nb = vd::join_buckets<" << S << ">(words[0]);\n";
		k << "  if (blockIdx.x == 0 && threadIdx.x == 0) { words[1] = nb - 1; }\n";
		k << "  const uint64_t nslots = nb * vd::slots_per_bucket<" << S << ">();\n";
		k << "  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nslots; i += (uint64_t)gridDim.x * blockDim.x) {\n";
		k << "    jt[i].key = 0; jt[i].pay = 0;\n  }\n}\n\n";
		k << "extern \"C\" __global__ void __launch_bounds__(256) " << name << "_insert(const VcParams p) {\n";
		k << "  unsigned long long* const words = " << words << ";\n";
		k << "  " << S << "* const jt = " << table << ";\n";
		k << "  const " << KT << "* const skeys = " << Pptr(jd.stage_keys, "const " + KT + "*") << ";\n";
		k << "  const " << PT << "* const spay = " << Pptr(jd.stage_pay, "const " + PT + "*") << ";\n";
		k << "  const uint64_t* const shash = " << Pptr(stage_hash(jd), "const uint64_t*") << ";\n";
		k << "  unsigned* const err = (unsigned*)p.v[" << err_slot << "];\n";
		k << "  const uint64_t cnt = words[0];\n";
		k << "  const uint64_t bmask = vd::join_buckets<" << S << ">(cnt) - 1;\n";
		k << "  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (uint64_t)gridDim.x * blockDim.x) {\n";
		k << "    vd::join_insert(jt, bmask, shash[i], skeys[i], spay[i], err);\n  }\n}\n\n";
		return k.str();
	}

	/* group extraction: rows with count > 0, keys unpacked, visible aggregates */
	std::string gen_extract() {
		Sink& s = p.sink;
		std::ostringstream k;
		k << "extern \"C\" __global__ void __launch_bounds__(256) " << name << "_extract(const VcParams p) {\n";
		k << "  int64_t* const out = " << Pptr(plan_out, "int64_t*") << ";\n";
		k << "  const int64_t ocap = " << P((unsigned long long)plan_out_cap) << ";\n";
		k << "  unsigned long long* const ocount = " << Pptr(out_count(), "unsigned long long*") << ";\n";
		k << "  const unsigned long long* const g = " << Pptr(s_dev(), "const unsigned long long*") << ";\n";
		const int W = s.kind == Sink::AggHash ? 1 + A() : A();
		const int off = s.kind == Sink::AggHash ? 1 : 0;
		int64_t nslots = s.kind == Sink::AggGlobal ? 1 : s.kind == Sink::AggDense ? (int64_t)s.domain : s_cap();
		k << "  const int64_t nslots = " << P((unsigned long long)nslots) << ";\n";
		k << "  const int64_t stride = (int64_t)gridDim.x * blockDim.x;\n";
		k << "  for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < nslots; base += stride) {\n";
		k << "    const int64_t i = base + (threadIdx.x & 31);\n";
		k << "    bool take = false;\n";
		k << "    if (i < nslots) {\n";
		if (s.kind == Sink::AggHash) {
			k << "      take = g[i * " << W << "] != 0ull && (int64_t)g[i * " << W << " + 1 + " << s.count_idx << "] > 0;\n";
		} else {
			k << "      take = (int64_t)g[i * " << W << " + " << s.count_idx << "] > 0;\n";
		}
		k << "    }\n";
		k << "    const int64_t pos = vd::warp_append(ocount, take);\n";
		k << "    if (take && pos < ocap) {\n";
		int col = 0;
		for (size_t kk = 0; kk < s.keys.size(); kk++, col++) {
			const std::string lo = P((unsigned long long)(int64_t)s.keys[kk]->b.lo);
			if (s.kind == Sink::AggDense) {
				const int64_t range = (int64_t)(s.keys[kk]->b.hi - s.keys[kk]->b.lo + 1);
				k << "      out[" << col << " * ocap + pos] = " << lo << " + (i / " << P((unsigned long long)s.key_radix[kk])
				  << ") % " << P((unsigned long long)range) << ";\n";
			} else {
				const int bits = (kk + 1 < s.keys.size() ? s.key_shift[kk + 1] : s.key_bits) - s.key_shift[kk];
				const unsigned long long mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1ull);
				k << "      out[" << col << " * ocap + pos] = " << lo << " + (int64_t)(((g[i * " << W << "] - 1ull) >> "
				  << P((unsigned long long)s.key_shift[kk]) << ") & " << Pu(mask) << ");\n";
			}
		}
		for (int a = 0; a < A(); a++) {
			if (!s.aggs[a].visible) {
				continue;
			}
			k << "      out[" << col << " * ocap + pos] = (int64_t)g[i * " << W << " + " << off + a << "];\n";
			col++;
		}
		k << "    }\n  }\n}\n\n";
		return k.str();
	}

	/* state accessors, set by the runtime before generation */
	void* s_dev_ptr = nullptr;
	int64_t s_cap_val = 0;
	void* stage_hash_ptr = nullptr;
	unsigned long long* out_count_ptr = nullptr;
	void* plan_out = nullptr;
	int64_t plan_out_cap = 0;
	size_t err_slot = 1;
	bool dense_in_smem = false;
	int cache_slots = 0;

	void* s_dev() { return s_dev_ptr; }
	int64_t s_cap() { return s_cap_val; }
	void* stage_hash(JoinDesc&) { return stage_hash_ptr; }
	unsigned long long* out_count() { return out_count_ptr; }
};

} // namespace

GeneratedCode generate_cuda(LoweredPlan& plan, const Flavor& fl, std::vector<PipeDeviceState>& st,
	void* out, int64_t out_cap, unsigned long long* out_count, std::vector<std::vector<unsigned long long>>& params)
{
	GeneratedCode gc;
	std::ostringstream src;
	src << "#include \"voila_device.cuh\"\n";
	params.assign(plan.pipes.size(), {});
	for (auto& p : plan.pipes) {
		auto& prm = params[p.id];
		PipeGen g(p, plan, fl, prm);
		g.s_dev_ptr = st[p.id].sink_dev;
		g.s_cap_val = st[p.id].sink_cap;
		g.stage_hash_ptr = st[p.id].stage_hash;
		g.out_count_ptr = out_count;
		g.plan_out = out;
		g.plan_out_cap = out_cap;
		size_t smem = 0;
		std::string main = g.gen_main(smem);
		std::string extra;
		if (p.sink.kind == Sink::JoinBuild) {
			extra = g.gen_join_build();
		} else if (p.sink.kind == Sink::AggGlobal || p.sink.kind == Sink::AggDense || p.sink.kind == Sink::AggHash) {
			extra = g.gen_extract();
		}
		src << "#define VcParams VcParams" << p.id << "\n";
		src << "struct VcParams" << p.id << " { unsigned long long v[" << std::max<size_t>(prm.size(), 1) << "]; };\n";
		src << main << extra;
		src << "#undef VcParams\n\n";

		Launch m;
		m.kernel = g.name + "_main";
		m.pipe = p.id;
		m.stage = 0;
		m.smem = smem;
		m.threads = fl.threads;
		const int64_t tile = (int64_t)fl.threads * fl.rows;
		m.grid_items = (p.rows + tile - 1) / tile;
		m.dominant = p.id == plan.result_pipe;
		if (p.sink.kind == Sink::JoinBuild) {
			gc.launches.push_back(m);
			Launch c;
			c.kernel = g.name + "_clear";
			c.pipe = p.id;
			c.stage = 1;
			c.threads = 256;
			c.grid_items = 0;
			gc.launches.push_back(c);
			Launch ins = c;
			ins.kernel = g.name + "_insert";
			ins.stage = 2;
			gc.launches.push_back(ins);
		} else {
			gc.launches.push_back(m);
			if (p.sink.kind != Sink::Emit) {
				Launch e;
				e.kernel = g.name + "_extract";
				e.pipe = p.id;
				e.stage = 1;
				e.threads = 256;
				const int64_t nslots = p.sink.kind == Sink::AggGlobal ? 1
					: p.sink.kind == Sink::AggDense ? (int64_t)p.sink.domain : st[p.id].sink_cap;
				e.grid_items = (nslots + 255) / 256;
				gc.launches.push_back(e);
			}
		}
	}
	gc.source = src.str();
	return gc;
}

} // namespace vc
