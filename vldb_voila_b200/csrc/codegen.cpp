/*
 * CUDA code generator: one fused kernel per lowered pipeline.
 *
 * This is the CUDA counterpart of the reference's per-pipeline code generators
 * (cg_hyper.cpp gen_pipeline :804-845, cg_vector.cpp :793-923): where those emit a
 * tuple-at-a-time loop or a chain of vector primitives, this emits a CUDA kernel in which
 * every thread owns `rows` consecutive rows of a tile, evaluates the pipeline's filters and
 * probes for all of them (op-major, so independent hash-table loads overlap) and feeds its
 * sink.  Column tiles arrive either by vector loads (load=ldg) or through a multi-stage
 * shared-memory ring filled by bulk asynchronous copies (load=tma).  Per pipeline sink:
 *
 *   JoinBuild  direct: filter + insert into a table sized for every build row
 *              staged: materialise (write/write_pos, relalg_translator.cpp:828-907) with a
 *                      block-aggregated append, then clear + insert sized by the count
 *                      (bucket_build / build_index, runtime_struct.cpp:1283-1324)
 *   AggGlobal  registers -> block reduction -> one atomic per CTA (aggr_gsum/gcount); the
 *              last CTA publishes the row
 *   AggDense   shared-memory slots over the key domain with warp-combined updates, merged
 *              into a global slot array; the last CTA emits slots with count > 0
 *   AggHash    global open-addressing group table with warp-combined leader updates and an
 *              optional per-CTA shared-memory cache for hot keys; separate extract kernel
 *   Emit       block-aggregated append of the selected rows
 *
 * The source depends only on the plan's shape (column types, operators, aggregate count)
 * and the flavor knobs; every data-dependent number (row counts, constants, key ranges,
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
	case VC_TYPE_STR: return "int32_t"; /* dictionary codes */
	default: return "int64_t";
	}
}

static int type_bytes(int t)
{
	return vc_gen_type_size(t);
}

static int64_t pow2_at_least(int64_t x)
{
	int64_t p = 1;
	while (p < x) {
		p <<= 1;
	}
	return p;
}

/* bits of hi - lo for a value of bounds b (64 when the span does not fit 64 bits) */
static int span_bits(const Bounds& b)
{
	const __int128 span = b.hi - b.lo;
	if (span < 0 || span >= ((__int128)1 << 64)) {
		return 64;
	}
	int bits = 0;
	for (unsigned __int128 x = (unsigned __int128)span; x; x >>= 1) {
		bits++;
	}
	return std::max(bits, 1);
}

PartPlan part_plan(const Pipeline& p, const LoweredPlan& plan, const Flavor& f, int sms)
{
	PartPlan pp;
	const Sink& s = p.sink;
	/* aggr=auto partitions group-bys whose groups bound passes 2^18 (a global table of
	 * several MiB and more, where random atomics into it dominate) */
	const bool wanted = f.aggr == "part" || (f.aggr == "auto" && s.groups_bound >= (int64_t)1 << 18);
	if (!wanted || s.kind != Sink::AggHash || s.key_bits > 31 || s.count_idx < 0) {
		return PartPlan();
	}
	/* record: the packed key in the low bits of word 0, then each summed value (minus its
	 * lower bound) in a field of its span's width; a field never straddles two words */
	int word = 0, off = s.key_bits;
	pp.rec_word.assign(s.aggs.size(), -1);
	pp.rec_off.assign(s.aggs.size(), 0);
	for (size_t a = 0; a < s.aggs.size(); a++) {
		if (s.aggs[a].count) {
			continue;
		}
		const int bits = span_bits(s.aggs[a].arg->b);
		if (bits >= 64) {
			return PartPlan();
		}
		if (off + bits > 64) {
			word++;
			off = 0;
		}
		if (word >= 2) {
			return PartPlan();
		}
		pp.rec_word[a] = word;
		pp.rec_off[a] = off;
		off += bits;
	}
	pp.rec_words = word + 1;
	const int W = s.nwords;
	/* a partition's table: the most slots whose keys and words fit 96 KiB */
	int S = 16384;
	while (S > 1024 && (size_t)S * (4 + 8 * (size_t)W) > 96 * 1024) {
		S >>= 1;
	}
	if ((size_t)S * (4 + 8 * (size_t)W) > 96 * 1024) {
		return PartPlan();
	}
	const int64_t groups = std::max<int64_t>(s.groups_bound, 1);
	int64_t P = f.parts ? f.parts : std::min<int64_t>(2048, std::max<int64_t>(16, pow2_at_least((groups * 2 + S - 1) / S)));
	/* on average a partition's table is at most three quarters full */
	if (groups > P * S * 3 / 4) {
		return PartPlan();
	}
	pp.P = (int)P;
	while ((1 << pp.log2P) < pp.P) {
		pp.log2P++;
	}
	pp.S = S;
	/* the histogram and scatter passes run the same grid: at most the CTAs that the threads
	 * of a CTA allow per SM */
	pp.max_ctas = (int64_t)sms * std::max(1, 2048 / f.threads);
	pp.smem1 = (size_t)P * 4;
	bool joinn = false;
	for (auto& op : p.ops) {
		joinn = joinn || (op.kind == Op::Probe && !plan.joins[op.join].join01);
	}
	const int64_t rows = std::max<int64_t>(p.rows, 1);
	pp.cap = joinn ? 4 * rows + (1 << 20) : rows;
	if (pp.cap >= (int64_t)UINT32_MAX) {
		return PartPlan(); /* record positions are 32-bit */
	}
	pp.R = std::max<int64_t>(4 * (int64_t)S, (pp.cap + 2047) / 2048);
	pp.max_items = P + pp.cap / pp.R + 1;
	/* a split item leaves at most min(S, its records) groups; split items hold at least R / 2
	 * records each */
	pp.scratch = std::min<int64_t>(pp.cap, (2 * pp.cap / pp.R + 1) * S) + S;
	pp.smem2 = (size_t)S * 4 + (size_t)S * W * 8 + (size_t)P * 12 + (size_t)P * 8;
	pp.smem2 = (pp.smem2 + 15) & ~(size_t)15;
	return pp;
}

namespace {

struct PipeGen {
	Pipeline& p;
	LoweredPlan& plan;
	const Flavor& fl;
	const PipeDeviceState& st;
	const QueryDeviceState& qs;
	std::vector<unsigned long long>& params;
	std::ostringstream o;
	std::string name;
	int V;
	int T;
	size_t smem_sink = 0;      /* dynamic shared memory used by the sink */
	size_t smem_total = 0;
	int cache_slots = 0;
	bool dense_in_smem = false;
	int replicas = 1;          /* copies of the dense slot array (per warp or per group of warps) */
	bool leader_plain = false; /* each warp owns a copy: group leaders update it without atomics */
	std::map<const BExpr*, int> const_slot; /* parameter slot of each constant node */
	bool private_acc = false;  /* per-thread private accumulators (lowcard=private) */
	int kGmax = 8;             /* distinct groups per block held in private accumulators (pgroups) */
	bool regs_acc = false;     /* per-thread packed accumulators (lowcard=regs|packed) */
	bool regs_smem = false;    /* lowcard=packed: the packed words live in shared memory, one
	                            * column per thread, indexed by the row's code */
	int regs_tiles = 1;        /* tiles a thread sums into its registers between two flushes */
	int regs_words = 0;        /* packed 64-bit words per group */
	std::vector<int> rg_word, rg_shift, rg_bits; /* aggregate a's field, wide enough for a flush's rows */
	static constexpr int kExtractK = 4; /* slot groups per warp step of the group extraction */

	PipeGen(Pipeline& pp, LoweredPlan& pl, const Flavor& f, const PipeDeviceState& s, const QueryDeviceState& q,
		std::vector<unsigned long long>& prm)
		: p(pp), plan(pl), fl(f), st(s), qs(q), params(prm), V(f.rows), T(f.threads), kGmax(f.private_groups) {
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
		case BExpr::Const: {
			/* one slot per constant node and generation (the plan may be generated again,
			 * e.g. for a batch, with a different parameter layout) */
			auto it = const_slot.find(e.get());
			if (it == const_slot.end()) {
				params.push_back((unsigned long long)e->cval);
				it = const_slot.emplace(e.get(), (int)params.size() - 1).first;
			}
			return "((int64_t)p.v[" + std::to_string(it->second) + "])";
		}
		case BExpr::ProbeOut:
			return "pay" + std::to_string(e->probe) + "_" + std::to_string(e->pidx) + "[" + v + "]";
		case BExpr::Fun: {
			static const std::map<std::string, std::string> ops = {
				{"add", "+"}, {"sub", "-"}, {"mul", "*"}, {"lt", "<"}, {"le", "<="}, {"gt", ">"},
				{"ge", ">="}, {"eq", "=="}, {"ne", "!="}, {"and", "&&"}, {"or", "||"}};
			if (e->fn == "inset") {
				const CodeBitmap& bm = plan.bitmaps[(size_t)e->aux];
				return "vd::code_in(" + Pptr(bm.dev, "const unsigned*") + ", (int64_t)(" + expr(e->args[0], v) + ") - " +
					P((unsigned long long)bm.lo) + ", " + P((unsigned long long)(bm.bits.size() * 32)) + ")";
			}
			if (e->fn == "extract_year") {
				return "((int64_t)vd::julian_year((uint32_t)(" + expr(e->args[0], v) + ")))";
			}
			if (e->fn == "shr") {
				return "((int64_t)(" + expr(e->args[0], v) + ") >> " + std::to_string(e->args[1]->cval) + ")";
			}
			if (e->fn == "lowbits") {
				const unsigned long long m = (1ull << e->args[1]->cval) - 1ull;
				return "((int64_t)((uint64_t)(" + expr(e->args[0], v) + ") & " + std::to_string(m) + "ull))";
			}
			if (e->fn == "mul" && fits32(e->args[0]->b) && fits32(e->args[1]->b)) {
				return "vd::mulw(" + expr(e->args[0], v) + ", " + expr(e->args[1], v) + ")";
			}
			return "(" + expr(e->args[0], v) + " " + ops.at(e->fn) + " " + expr(e->args[1], v) + ")";
		}
		}
		return "0";
	}

	static bool fits32(const Bounds& b) {
		return b.lo >= (__int128)INT32_MIN && b.hi <= (__int128)INT32_MAX;
	}

	int A() const { return (int)p.sink.aggs.size(); }
	bool part_hist = false;    /* generating the histogram pass of a partitioned group-by */
	/* compaction within each warp (no block barriers): when the rest of the pipeline needs no
	 * block-wide collectives (appending sinks, JoinN loops over an appending sink), and no
	 * column is read in place from host memory -- there a block's flush, whose warps each take
	 * consecutive survivors of one stretch of rows, makes fewer PCIe requests per gather */
	bool warp_compact() const {
		for (auto& c : p.cols) {
			if (c.host) {
				return false;
			}
		}
		return !sink_block_collective();
	}
	/* survivors each thread takes per pass of a compaction flush (gathers in flight) */
	int FV() const { return fl.flush_rows; }
	/* partitioned aggregation (aggr=part) of a standalone pipeline */
	bool part() const { return st.part.P > 0 && !item; }
	std::string rec_type() const { return st.part.rec_words == 2 ? "ulonglong2" : "unsigned long long"; }
	/* stored key width of the split hash group table */
	/* hash group-by with a per-CTA shared-memory cache (aggr=cache, or aggr=dcache and
	 * aggr=auto over a direct table) */
	bool gcache() const { return fl.aggr == "cache" || fl.aggr == "dcache" || (fl.aggr == "auto" && gdirect()); }
	/* the group table is indexed by the packed key (aggr=direct|dcache): no keys, no probes */
	bool gdirect() const { return st.sink_direct; }
	int gkey_bytes() const { return p.sink.key_bits <= 31 ? 4 : 8; }
	std::string gkey_type() const { return p.sink.key_bits <= 31 ? "uint32_t" : "uint64_t"; }

	/* bits of value - lo for one row of aggregate a (the per-row span of the warp pre-sum) */
	/* Packs every aggregate's sum over R rows of one thread (value minus lower bound; the
	 * count) into bit fields of 64-bit words, first fit by decreasing width.  Returns the
	 * number of words, or 0 when a field would not fit a word. */
	int regs_pack(int64_t R, std::vector<int>& word, std::vector<int>& shift, std::vector<int>& bits) const {
		int rb = 0;
		for (int64_t x = R; x; x >>= 1) {
			rb++;
		}
		const int n = A();
		word.assign(n, 0);
		shift.assign(n, 0);
		bits.assign(n, 0);
		std::vector<int> order(n);
		for (int a = 0; a < n; a++) {
			order[a] = a;
			bits[a] = (p.sink.aggs[a].count ? 0 : row_bits(a)) + rb;
			if (bits[a] > 64) {
				return 0;
			}
		}
		std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return bits[x] > bits[y]; });
		std::vector<int> used;
		for (int a : order) {
			size_t w = 0;
			while (w < used.size() && used[w] + bits[a] > 64) {
				w++;
			}
			if (w == used.size()) {
				used.push_back(0);
			}
			word[a] = (int)w;
			shift[a] = used[w];
			used[w] += bits[a];
		}
		return (int)used.size();
	}

	/* lowcard=regs|packed: the flush interval F (tiles) and the field layout.  Per row, a
	 * thread adds its words: about 2.5 instructions per word and code under regs (every code's
	 * words, under a select), about 5 per word under packed (a shared-memory read-modify-write
	 * at the row's code); a warp's flush costs about 46 instructions per code and covers F·rows
	 * rows of each lane.  F minimises the sum (wider fields, more words, fewer flushes). */
	bool plan_regs() {
		std::vector<int> w, s, b;
		double best = 1e30;
		bool found = false;
		for (int F = 1; F <= 64; F <<= 1) {
			const int64_t R = (int64_t)F * V;
			const int wf = regs_pack(R, w, s, b);
			/* regs: at most 16 words (32 registers) of accumulators per thread; packed: at most
			 * 64 KiB of shared memory per CTA */
			if (wf == 0 || (!regs_smem && kGmax * wf > 16) || (regs_smem && (size_t)kGmax * wf * T * 8 > 64 * 1024)) {
				continue;
			}
			const double per_row = (regs_smem ? 5.0 * wf : 2.5 * kGmax * wf) + 46.0 * kGmax / (double)R;
			if (per_row < best) {
				best = per_row;
				found = true;
				regs_tiles = F;
				regs_words = wf;
				rg_word = w;
				rg_shift = s;
				rg_bits = b;
			}
		}
		return found;
	}

	int row_bits(int a) const {
		const auto& ag = p.sink.aggs[a];
		const __int128 span = ag.arg->b.hi - ag.arg->b.lo;
		if (span < 0 || span >= ((__int128)1 << 64)) {
			return 64;
		}
		int bits = 0;
		for (unsigned __int128 x = (unsigned __int128)span; x; x >>= 1) {
			bits++;
		}
		return std::max(bits, 1);
	}

	/* One field of a warp pre-sum: a lane's biased (non-negative) value of `bits` bits, summed
	 * into bit `shift` of accumulator word `word`; a count field sums one per lane. */
	struct PresumField {
		std::string val;
		int word, shift, bits;
		bool count;
	};

	/*
	 * Warp pre-aggregation into packed accumulator words w[W].  Lanes with the same group key
	 * (__match_any_sync of `key`, a sentinel on dead lanes) form a group; `lead` marks each
	 * group's lowest live lane, which updates the table for the group.  A single-lane group
	 * keeps its own values.  Groups of several lanes are summed one after another with
	 * full-warp redux.sync (lanes outside the group add zero): redux.sync with each group's
	 * own member mask would be executed once per distinct mask, so a warp of distinct keys
	 * would pay for 32 serialised reductions; this way it pays for none.
	 */
	void emit_presum(std::ostream& k, const std::string& ind, const std::string& key, const std::string& live,
		const std::vector<PresumField>& f, int W) {
		k << ind << "const unsigned gm = __match_any_sync(0xffffffffu, " << key << ");\n";
		k << ind << "const bool lead = (" << live << ") && (gm & vd::lanemask_lt()) == 0u;\n";
		for (size_t i = 0; i < f.size(); i++) {
			if (!f[i].count) {
				k << ind << "const uint64_t fv" << i << " = (" << live << ") ? (uint64_t)(" << f[i].val << ") : 0ull;\n";
			}
		}
		k << ind << "uint64_t w[" << W << "] = {";
		for (int i = 0; i < W; i++) {
			k << (i ? ", " : "") << "0ull";
		}
		k << "};\n";
		for (size_t i = 0; i < f.size(); i++) {
			if (f[i].count) {
				k << ind << "w[" << f[i].word << "] += (uint64_t)((" << live << ") ? 1u : 0u) << " << f[i].shift << ";\n";
			} else {
				k << ind << "w[" << f[i].word << "] += fv" << i << " << " << f[i].shift << ";\n";
			}
		}
		k << ind << "unsigned multi = __ballot_sync(0xffffffffu, lead && (gm & (gm - 1u)) != 0u);\n";
		k << ind << "while (multi) {\n";
		k << ind << "  const int gl = __ffs(multi) - 1;\n";
		k << ind << "  multi &= multi - 1u;\n";
		k << ind << "  const unsigned gg = __shfl_sync(0xffffffffu, gm, gl);\n";
		k << ind << "  const bool gin = ((gg >> vd::lane_id()) & 1u) != 0u;\n";
		k << ind << "  uint64_t g[" << W << "] = {";
		for (int i = 0; i < W; i++) {
			k << (i ? ", " : "") << "0ull";
		}
		k << "};\n";
		for (size_t i = 0; i < f.size(); i++) {
			if (f[i].count) {
				k << ind << "  g[" << f[i].word << "] += (uint64_t)__popc(gg) << " << f[i].shift << ";\n";
			} else {
				k << ind << "  g[" << f[i].word << "] += vd::group_sum_u<" << f[i].bits << ">(0xffffffffu, gin ? fv" << i
				  << " : 0ull) << " << f[i].shift << ";\n";
			}
		}
		k << ind << "  if ((int)vd::lane_id() == gl) {\n";
		k << ind << "#pragma unroll\n" << ind << "    for (int a = 0; a < " << W << "; a++) { w[a] = g[a]; }\n";
		k << ind << "  }\n";
		k << ind << "}\n";
	}

	/* the sink's aggregates as pre-sum fields of the packed accumulator words, values at row v */
	std::vector<PresumField> sink_fields(const std::string& v) {
		const Sink& s = p.sink;
		std::vector<PresumField> f;
		for (int a = 0; a < A(); a++) {
			const auto& ag = s.aggs[a];
			if (ag.count) {
				f.push_back({"", s.agg_word[a], s.agg_shift[a], 0, true});
				continue;
			}
			const std::string lo = P((unsigned long long)(int64_t)ag.arg->b.lo);
			f.push_back({"(uint64_t)(" + expr(ag.arg, v) + ") - (uint64_t)" + lo, s.agg_word[a], s.agg_shift[a], row_bits(a), false});
		}
		return f;
	}

	/* Warp pre-aggregation into packed accumulator words for row v (see emit_presum). */
	void emit_packed_words(const std::string& key, const std::string& v) {
		emit_presum(o, "      ", key, "act[" + v + "]", sink_fields(v), p.sink.nwords);
	}

	/* Warp pre-aggregation of one row per lane into vals[] (dense slots): lanes holding the
	 * same slot (`key`, a sentinel on inactive lanes) form a group whose lowest active lane
	 * (`lead`) ends up with the group's sums; a single-lane group keeps its own values, and
	 * groups of several lanes are summed one after another with full-warp redux.sync on the
	 * values biased by their lower bounds (non-negative, of known bit width). */
	void emit_group_reduce(const std::string& key) {
		o << "      const unsigned gm = __match_any_sync(0xffffffffu, " << key << ");\n";
		o << "      const bool lead = act[v] && (gm & vd::lanemask_lt()) == 0u;\n";
		std::vector<std::string> lo(A());
		for (int a = 0; a < A(); a++) {
			const auto& ag = p.sink.aggs[a];
			if (!ag.count) {
				lo[a] = P((unsigned long long)(int64_t)ag.arg->b.lo);
				o << "      const uint64_t fv" << a << " = act[v] ? (uint64_t)vals[" << a << "] - (uint64_t)" << lo[a]
				  << " : 0ull;\n";
			}
		}
		o << "      unsigned multi = __ballot_sync(0xffffffffu, lead && (gm & (gm - 1u)) != 0u);\n";
		o << "      while (multi) {\n";
		o << "        const int gl = __ffs(multi) - 1;\n";
		o << "        multi &= multi - 1u;\n";
		o << "        const unsigned gg = __shfl_sync(0xffffffffu, gm, gl);\n";
		o << "        const bool gin = ((gg >> vd::lane_id()) & 1u) != 0u;\n";
		o << "        const uint64_t gn = (uint64_t)__popc(gg);\n";
		for (int a = 0; a < A(); a++) {
			const auto& ag = p.sink.aggs[a];
			if (ag.count) {
				o << "        if ((int)vd::lane_id() == gl) { vals[" << a << "] = (int64_t)gn; }\n";
				continue;
			}
			o << "        const uint64_t gs" << a << " = vd::group_sum_u<" << row_bits(a) << ">(0xffffffffu, gin ? fv" << a
			  << " : 0ull);\n";
			o << "        if ((int)vd::lane_id() == gl) { vals[" << a << "] = (int64_t)(gs" << a << " + (uint64_t)" << lo[a]
			  << " * gn); }\n";
		}
		o << "      }\n";
	}

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

	/* hash that picks table positions: voila_hash chain of the raw keys (hash=voila) or
	 * the finalizer-mixed bit-packed key (hash=mix) */
	std::string table_hash(const std::vector<BExprP>& keys, const std::string& packed, int bits,
		const std::string& v) {
		if (fl.hash == "voila") {
			return key_hash(keys, v);
		}
		return bits <= 32 ? "vd::mix_hash32((uint32_t)(" + packed + "))" : "vd::mix_hash64(" + packed + ")";
	}

	std::string join_slot_type(const JoinDesc& jd) {
		return std::string("vd::JoinSlot<") + (jd.key64 ? "uint64_t" : "uint32_t") + ", " +
			(jd.pay64 ? "uint64_t" : "uint32_t") + ">";
	}

	/* ------------------------------------------------------------ main kernel ------ */

	/* item mode: the pipeline body becomes a device function over a tile range [t_begin,
	 * t_end) that the persistent batch kernel calls; parameters come from a pool in global
	 * memory instead of the kernel parameter space */
	bool item = false;
	std::string tstart() const { return item ? "t_begin" : "(int64_t)blockIdx.x"; }
	/* item k of a pipeline's nitems items takes tiles k, k + nitems, ...: items that run at
	 * the same time read neighbouring tiles, as the CTAs of a standalone launch do */
	std::string tstep() const { return item ? "nitems" : "(int64_t)gridDim.x"; }
	std::string tend() const { return item ? "tlim" : "ntiles"; }
	std::string blocks_total() const { return item ? "(unsigned long long)nitems" : "(unsigned long long)gridDim.x"; }

	void fn_header(const std::string& suffix) {
		if (item) {
			o << "__device__ __noinline__ void " << name << suffix
			  << "(const unsigned long long* __restrict__ pv, int64_t t_begin, int64_t t_end, int64_t nitems) {\n";
			o << "  const struct { const unsigned long long* __restrict__ v; } p = {pv};\n";
			o << "  (void)nitems;\n";
		} else {
			o << "extern \"C\" __global__ void __launch_bounds__(" << T
			  << (fl.min_ctas > 0 ? ", " + std::to_string(fl.min_ctas) : std::string()) << ") " << name << suffix
			  << "(const VcParams p) {\n";
			o << "  vd::pdl_launch_dependents();\n";
		}
	}

	/* before the first access to anything an earlier kernel of the query writes (tables,
	 * accumulators, results); the pipeline's own base columns may be read before it */
	void emit_pdl_wait() {
		if (!item) {
			o << "  vd::pdl_wait();\n";
		}
	}

	std::string gen_main() {
		fn_header(part_hist ? "_hist" : "_main");
		if (p.source_inter >= 0) {
			/* the rows come from an earlier pipeline of the query: wait for it before reading
			 * the row count (or any column) */
			const InterTable& it = plan.inters[p.source_inter];
			emit_pdl_wait();
			o << "  const int64_t n = min((int64_t)__ldcg(" << Pptr(it.count, "const unsigned long long*") << "), "
			  << P((unsigned long long)it.cap) << ");\n";
		} else {
			o << "  const int64_t n = " << P((unsigned long long)p.rows) << ";\n";
		}
		if (part_hist) {
			/* the histogram pass reads the same error word and column pointers as the main kernel */
			o << "  unsigned* const err = (unsigned*)p.v[" << p.err_slot << "];\n";
			for (size_t c = 0; c < p.cols.size(); c++) {
				o << "  const " << ctype(p.cols[c].type) << "* __restrict__ c" << c << " = (const "
				  << ctype(p.cols[c].type) << "*)p.v[" << p.col_slots[c] << "];\n";
			}
		} else {
			p.err_slot = (int)params.size();
			o << "  unsigned* const err = (unsigned*)p.v[" << params.size() << "];\n";
			params.push_back(0); /* error word, filled by the runtime */
			p.col_slots.clear();
			for (size_t c = 0; c < p.cols.size(); c++) {
				p.col_slots.push_back((int)params.size());
				o << "  const " << ctype(p.cols[c].type) << "* __restrict__ c" << c << " = (const "
				  << ctype(p.cols[c].type) << "*)p.v[" << params.size() << "];\n";
				params.push_back(0); /* column pointer, filled by the runtime */
			}
		}
		o << "  (void)err;\n";
		o << "  extern __shared__ __align__(128) unsigned char vd_smem[];\n";
		plan_phases();
		sink_prologue();
		o << "  const int64_t tile = (int64_t)" << T << " * " << V << ";\n";
		o << "  const int64_t ntiles = (n + tile - 1) / tile;\n";
		if (item) {
			o << "  const int64_t tlim = t_end < ntiles ? t_end : ntiles;\n";
		}

		emit_compaction_smem();
		bool any_eager = false;
		for (size_t c = 0; c < p.cols.size(); c++) {
			any_eager = any_eager || eager[c];
		}
		bool any_host = false; /* bulk copies do not read host-resident columns */
		for (auto& pc : p.cols) {
			any_host = any_host || pc.host;
		}
		const bool tma = fl.load == "tma" && any_eager && !item && !any_host;
		if (tma) {
			emit_pdl_wait();
			gen_tma_loop();
		} else if (fl.prefetch && any_eager) {
			/* register double buffering: the next tile's eager columns are in flight while
			 * this tile's probes and aggregation run */
			o << "  {\n";
			for (size_t c = 0; c < p.cols.size(); c++) {
				if (eager[c]) {
					o << "  " << ctype(p.cols[c].type) << " pf" << c << "[" << V << "];\n";
				}
			}
			o << "  int64_t t = " << tstart() << ";\n";
			o << "  if (t < " << tend() << ") {\n    const int64_t r0p = t * tile + (int64_t)threadIdx.x * " << V << ";\n";
			emit_load_cols("ldg", "pf", "r0p");
			o << "  }\n";
			/* the first tile's columns are in flight while the previous kernel finishes */
			emit_pdl_wait();
			o << "  for (; t < " << tend() << "; t += " << tstep() << ") {\n";
			emit_decl_cols(true, V);
			for (size_t c = 0; c < p.cols.size(); c++) {
				if (eager[c]) {
					o << "#pragma unroll\n    for (int v = 0; v < " << V << "; v++) { x" << c << "[v] = pf" << c << "[v]; }\n";
				}
			}
			o << "    {\n    const int64_t tn = t + " << tstep() << ";\n";
			o << "    if (tn < " << tend() << ") {\n    const int64_t r0p = tn * tile + (int64_t)threadIdx.x * " << V << ";\n";
			emit_load_cols("ldg", "pf", "r0p");
			o << "    }\n    }\n";
			emit_body("pre");
			o << "  }\n  }\n";
		} else {
			emit_pdl_wait();
			o << "  for (int64_t t = " << tstart() << "; t < " << tend() << "; t += " << tstep() << ") {\n";
			emit_body("ldg");
			o << "  }\n";
		}
		if (compact_at >= 0) {
			o << "  if (cpend > 0) { cflush(); }\n";
		}
		if (regs_acc) {
			o << "  rflush();\n";
		}
		sink_epilogue();
		o << "}\n\n";
		if (regs_acc) {
			o << "#undef racc\n";
		}
		smem_total = std::max(smem_total, smem_sink);
		return o.str();
	}

	/* tile bytes of all columns, each region 16-byte aligned */
	size_t tile_region(size_t c) {
		size_t off = 0;
		for (size_t i = 0; i < c; i++) {
			if (!eager[i]) {
				continue;
			}
			off += (size_t)T * V * type_bytes(p.cols[i].type);
			off = (off + 15) & ~(size_t)15;
		}
		return off;
	}

	/* The ring without block barriers, for bodies with no block-wide collectives: each stage
	 * has a full barrier (the bulk copies' bytes) and an empty barrier that every warp arrives
	 * on once it has read the stage; thread 0 refills the stage of the previous tile as soon as
	 * all warps have left it, so warps drift apart by up to the ring's depth instead of
	 * meeting at a barrier after every tile.  A wait that runs out sets the error word and
	 * the block's abort flag; each warp leaves the loop at its next tile (a warp-uniform
	 * vote), and thread 0 waits, bounded, for the copies still in flight. */
	void gen_tma_ring_decoupled() {
		const int S = fl.stages;
		const int NW = T / 32;
		const size_t tile_bytes = tile_region(p.cols.size());
		size_t base = (smem_sink + 127) & ~(size_t)127;
		const size_t bar_off = base + (size_t)S * tile_bytes;
		smem_total = bar_off + 16 * (size_t)S;
		o << "  unsigned char* const stages = vd_smem + " << base << ";\n";
		o << "  uint64_t* const full = (uint64_t*)(vd_smem + " << bar_off << ");\n";
		o << "  uint64_t* const empty = full + " << S << ";\n";
		o << "  __shared__ int tma_abort;\n";
		o << "  const int64_t nfull = n / tile;\n";
		o << "  const int64_t nmine = nfull > (int64_t)blockIdx.x ? (nfull - (int64_t)blockIdx.x + (int64_t)gridDim.x - 1) / "
		     "(int64_t)gridDim.x : 0;\n";
		o << "  if (threadIdx.x == 0) {\n";
		o << "    for (int s = 0; s < " << S << "; s++) { vd::mbar_init(&full[s], 1); vd::mbar_init(&empty[s], " << NW << "); }\n";
		o << "    vd::mbar_init_fence();\n    tma_abort = 0;\n";
		o << "  }\n  vd::block_sync();\n";
		o << "  auto issue = [&](int64_t j) {\n";
		o << "    const int64_t tj = (int64_t)blockIdx.x + j * (int64_t)gridDim.x;\n";
		o << "    const int s = (int)(j % " << S << ");\n";
		o << "    unsigned char* dst = stages + (size_t)s * " << tile_bytes << ";\n";
		o << "    vd::mbar_expect_tx(&full[s], " << tile_bytes_tx() << ");\n";
		for (size_t c = 0; c < p.cols.size(); c++) {
			if (!eager[c]) {
				continue;
			}
			const int tb = type_bytes(p.cols[c].type);
			o << "    vd::bulk_load(dst + " << tile_region(c) << ", c" << c << " + tj * tile, " << (size_t)T * V * tb
			  << "u, &full[s]);\n";
		}
		o << "  };\n";
		o << "  int64_t issued = 0;\n";
		o << "  if (threadIdx.x == 0) {\n";
		o << "    vd::fence_proxy_async();\n";
		o << "    for (; issued < " << S << " && issued < nmine; issued++) { issue(issued); }\n";
		o << "  }\n";
		o << "  int64_t i = 0;\n";
		o << "  for (; i < nmine; i++) {\n";
		o << "    if (threadIdx.x == 0 && i >= 1 && issued < nmine) {\n";
		o << "      const int64_t r = i - 1;\n";
		o << "      if (vd::mbar_wait(&empty[r % " << S << "], (uint32_t)((r / " << S << ") & 1))) {\n";
		o << "        vd::fence_proxy_async();\n        issue(issued);\n        issued++;\n";
		o << "      } else {\n        atomicOr(err, VD_ERR_WAIT_TIMEOUT);\n        *(volatile int*)&tma_abort = 1;\n      }\n";
		o << "    }\n";
		o << "    const int s = (int)(i % " << S << ");\n";
		o << "    const bool ok = vd::mbar_wait(&full[s], (uint32_t)((i / " << S << ") & 1));\n";
		o << "    if (!ok) { atomicOr(err, VD_ERR_WAIT_TIMEOUT); *(volatile int*)&tma_abort = 1; }\n";
		o << "    if (__any_sync(0xffffffffu, !ok || *(volatile int*)&tma_abort != 0)) { break; }\n";
		o << "    const int64_t t = (int64_t)blockIdx.x + i * (int64_t)gridDim.x;\n";
		o << "    const unsigned char* stage = stages + (size_t)s * " << tile_bytes << ";\n";
		emit_body("smem");
		o << "    __syncwarp();\n";
		o << "    if (vd::lane_id() == 0u) { vd::mbar_arrive(&empty[s]); }\n";
		o << "  }\n";
		/* after an abort: the copies issued but not consumed by thread 0's warp */
		o << "  if (threadIdx.x == 0) {\n";
		o << "    for (int64_t j = i; j < issued; j++) {\n";
		o << "      vd::mbar_wait(&full[j % " << S << "], (uint32_t)((j / " << S << ") & 1), 100000000ull);\n";
		o << "    }\n  }\n";
		o << "  vd::block_sync();\n";
		o << "  if (nfull < ntiles && (int64_t)blockIdx.x == nfull % (int64_t)gridDim.x) {\n";
		o << "    const int64_t t = nfull;\n";
		emit_body("ldg");
		o << "  }\n";
	}

	/* the body has no block barriers or block-wide votes (warp-level work only) */
	bool body_warp_only() const {
		return !sink_block_collective() && (compact_at < 0 || warp_compact());
	}

	void gen_tma_loop() {
		if (body_warp_only()) {
			gen_tma_ring_decoupled();
			return;
		}
		const int S = fl.stages;
		const size_t tile_bytes = tile_region(p.cols.size());
		size_t base = (smem_sink + 127) & ~(size_t)127;
		const size_t bar_off = base + (size_t)S * tile_bytes;
		smem_total = bar_off + 8 * (size_t)S;
		o << "  unsigned char* const stages = vd_smem + " << base << ";\n";
		o << "  uint64_t* const full = (uint64_t*)(vd_smem + " << bar_off << ");\n";
		o << "  const int64_t nfull = n / tile;\n";
		o << "  if (threadIdx.x == 0) {\n";
		o << "    for (int s = 0; s < " << S << "; s++) { vd::mbar_init(&full[s], 1); }\n";
		o << "    vd::mbar_init_fence();\n";
		o << "  }\n  vd::block_sync();\n";
		/* issue helper as a lambda */
		o << "  auto issue = [&](int64_t j) {\n";
		o << "    const int64_t tj = (int64_t)blockIdx.x + j * (int64_t)gridDim.x;\n";
		o << "    if (tj >= nfull) { return; }\n";
		o << "    const int s = (int)(j % " << S << ");\n";
		o << "    unsigned char* dst = stages + (size_t)s * " << tile_bytes << ";\n";
		o << "    vd::mbar_expect_tx(&full[s], " << tile_bytes_tx() << ");\n";
		for (size_t c = 0; c < p.cols.size(); c++) {
			if (!eager[c]) {
				continue;
			}
			const int tb = type_bytes(p.cols[c].type);
			o << "    vd::bulk_load(dst + " << tile_region(c) << ", c" << c << " + tj * tile, " << (size_t)T * V * tb
			  << "u, &full[s]);\n";
		}
		o << "  };\n";
		o << "  if (threadIdx.x == 0) {\n";
		o << "    vd::fence_proxy_async();\n";
		o << "    for (int j = 0; j < " << S - 1 << "; j++) { issue(j); }\n";
		o << "  }\n";
		o << "  bool timed_out = false;\n";
		o << "  int64_t i = 0;\n";
		o << "  for (;; i++) {\n";
		o << "    const int64_t t = (int64_t)blockIdx.x + i * (int64_t)gridDim.x;\n";
		o << "    if (t >= nfull) { break; }\n";
		o << "    if (threadIdx.x == 0) { vd::fence_proxy_async(); issue(i + " << S - 1 << "); }\n";
		o << "    const int s = (int)(i % " << S << ");\n";
		o << "    const bool ok = vd::mbar_wait(&full[s], (uint32_t)((i / " << S << ") & 1));\n";
		o << "    if (vd::block_any(!ok)) { timed_out = true; break; }\n";
		o << "    const unsigned char* stage = stages + (size_t)s * " << tile_bytes << ";\n";
		emit_body("smem");
		o << "    vd::block_sync();\n";
		o << "  }\n";
		o << "  if (timed_out) {\n";
		o << "    if (threadIdx.x == 0) {\n";
		o << "      atomicOr(err, VD_ERR_WAIT_TIMEOUT);\n";
		o << "      for (int64_t j = i; j < i + " << S - 1 << "; j++) {\n";
		o << "        if ((int64_t)blockIdx.x + j * (int64_t)gridDim.x < nfull) {\n";
		o << "          vd::mbar_wait(&full[j % " << S << "], (uint32_t)((j / " << S << ") & 1), 100000000ull);\n";
		o << "        }\n      }\n    }\n";
		o << "    vd::block_sync();\n";
		o << "  } else if (nfull < ntiles && (int64_t)blockIdx.x == nfull % (int64_t)gridDim.x) {\n";
		o << "    const int64_t t = nfull;\n";
		emit_body("ldg");
		o << "  }\n";
	}

	size_t tile_bytes_tx() {
		size_t b = 0;
		for (size_t c = 0; c < p.cols.size(); c++) {
			if (eager[c]) {
				b += (size_t)T * V * type_bytes(p.cols[c].type);
			}
		}
		return b;
	}

	/* ------------------------------------------------------------ column phases ---- */

	int compact_at = -1;              /* op index after which survivors are compacted */
	std::vector<bool> eager;          /* column loaded with the tile (else gathered after compaction) */
	std::vector<std::pair<int, int>> carried; /* (probe op, payload) values carried through compaction */

	static void cols_of(const BExprP& e, std::vector<bool>& used) {
		if (e->kind == BExpr::Col) {
			used[e->col] = true;
		}
		for (auto& a : e->args) {
			cols_of(a, used);
		}
	}
	static void payloads_of(const BExprP& e, std::vector<std::pair<int, int>>& out) {
		if (e->kind == BExpr::ProbeOut) {
			std::pair<int, int> k(e->probe, e->pidx);
			if (std::find(out.begin(), out.end(), k) == out.end()) {
				out.push_back(k);
			}
		}
		for (auto& a : e->args) {
			payloads_of(a, out);
		}
	}
	std::vector<BExprP> sink_exprs() {
		std::vector<BExprP> r;
		for (auto& k : p.sink.keys) r.push_back(k);
		if (part_hist) {
			return r;
		}
		for (auto& k : p.sink.pay) r.push_back(k);
		for (auto& a : p.sink.aggs) if (a.arg) r.push_back(a.arg);
		for (auto& k : p.sink.outs) r.push_back(k);
		return r;
	}

	bool has_join_n() const {
		for (auto& op : p.ops) {
			if (op.kind == Op::Probe && !plan.joins[op.join].join01) {
				return true;
			}
		}
		return false;
	}

	void plan_phases() {
		compact_at = has_join_n() ? -1 : fl.compact;
		if (compact_at == -2) {
			/* auto: after the first probe when more probes follow */
			compact_at = -1;
			for (size_t i = 0; i < p.ops.size(); i++) {
				if (p.ops[i].kind == Op::Probe) {
					for (size_t j = i + 1; j < p.ops.size(); j++) {
						if (p.ops[j].kind == Op::Probe) {
							compact_at = (int)i;
						}
					}
					break;
				}
			}
		}
		if (compact_at >= (int)p.ops.size()) {
			compact_at = -1;
		}
		eager.assign(p.cols.size(), compact_at < 0);
		carried.clear();
		if (compact_at < 0) {
			if (part_hist) {
				/* the histogram pass reads only what the ops and the group keys need */
				eager.assign(p.cols.size(), false);
				for (auto& op : p.ops) {
					if (op.pred) cols_of(op.pred, eager);
					for (auto& k : op.keys) cols_of(k, eager);
				}
				for (auto& k : p.sink.keys) cols_of(k, eager);
			}
			return;
		}
		for (int i = 0; i <= compact_at; i++) {
			const Op& op = p.ops[i];
			if (op.pred) cols_of(op.pred, eager);
			for (auto& k : op.keys) cols_of(k, eager);
		}
		std::vector<BExprP> later = sink_exprs();
		for (size_t i = compact_at + 1; i < p.ops.size(); i++) {
			if (p.ops[i].pred) later.push_back(p.ops[i].pred);
			for (auto& k : p.ops[i].keys) later.push_back(k);
		}
		for (auto& e : later) {
			payloads_of(e, carried);
		}
		carried.erase(std::remove_if(carried.begin(), carried.end(),
			[&](const std::pair<int, int>& c) { return c.first > compact_at; }), carried.end());
	}

	void emit_decl_cols(bool only_eager, int rows) {
		for (size_t c = 0; c < p.cols.size(); c++) {
			if (only_eager && !eager[c]) {
				continue;
			}
			o << "    " << ctype(p.cols[c].type) << " x" << c << "[" << rows << "];\n";
		}
	}

	/* template load mode of column c (vd::col_ld): 1 host-resident, 2 stream=noalloc, else 0 */
	std::string load_mode(size_t c) const {
		if (p.cols[c].host) {
			return ", 1";
		}
		return fl.stream == "noalloc" ? ", 2" : "";
	}

	void emit_load_cols(const std::string& src, const std::string& dst, const std::string& r0) {
		for (size_t c = 0; c < p.cols.size(); c++) {
			if (!eager[c]) {
				continue;
			}
			const char* ct = ctype(p.cols[c].type);
			if (src == "smem") {
				o << "    vd::load_rows_smem<" << ct << ", " << V << ">((const " << ct << "*)(stage + " << tile_region(c)
				  << ") + threadIdx.x * " << V << ", " << dst << c << ");\n";
			} else {
				o << "    vd::load_rows<" << ct << ", " << V << load_mode(c) << ">(c" << c << ", " << r0
				  << ", n, " << dst << c << ");\n";
			}
		}
	}

	void emit_ops(int from, int to) {
		for (int i = from; i < to; i++) {
			const Op& op = p.ops[i];
			if (op.kind == Op::Filter) {
				o << "#pragma unroll\n    for (int v = 0; v < " << V << "; v++) { act[v] = act[v] && "
				  << expr(op.pred, "v") << "; }\n";
			} else {
				gen_probe(i, op);
			}
		}
	}

	/* lazy gathers (the compaction flush): column c is loaded before op lazy_first_use[c] */
	bool lazy_rows = false;
	std::vector<int> lazy_first_use;

	void emit_lazy_loads(int at) {
		if (!lazy_rows) {
			return;
		}
		for (size_t c = 0; c < p.cols.size(); c++) {
			if (lazy_first_use[c] == at) {
				o << "#pragma unroll\n      for (int v = 0; v < " << V << "; v++) { if (act[v]) { x" << c << "[v] = vd::load_one<"
				  << ctype(p.cols[c].type) << load_mode(c) << ">(c" << c << ", row[v]); } }\n";
			}
		}
	}

	/* ops [from, end) and the sink; a JoinN probe turns the rest of the pipeline into the body
	 * of its loop over matches */
	void emit_rest(int from) {
		for (int i = from; i < (int)p.ops.size(); i++) {
			const Op& op = p.ops[i];
			emit_lazy_loads(i);
			if (op.kind == Op::Probe && !plan.joins[op.join].join01) {
				gen_probe_n(i, op);
				return;
			}
			emit_ops(i, i + 1);
		}
		emit_lazy_loads((int)p.ops.size());
		sink_row();
	}

	/* sinks whose rows use block-wide collectives (appends): loops around them must be
	 * uniform over the block, not just the warp */
	bool sink_block_collective() const {
		return p.sink.kind == Sink::Emit ||
			(p.sink.kind == Sink::JoinBuild && !plan.joins[p.sink.join].direct && !plan.joins[p.sink.join].dense);
	}

	/*
	 * JoinN probe (relalg_translator.cpp:1032-1042 without the Join01 exit; bucket_next,
	 * kernel_generator.py:543-555): every build row with the probe row's key is a match and
	 * the rest of the pipeline runs once per match.  The table keeps duplicate keys in
	 * separate slots of the probe sequence, which ends at the first empty slot.  Each round
	 * of the loop gives every row at most one more match (act = has one); the loop runs
	 * while any row of the warp (or block, for appending sinks) still has slots to scan, so
	 * the warp-wide pre-aggregation of the sink sees converged warps.
	 */
	void gen_probe_n(int opi, const Op& op) {
		JoinDesc& jd = plan.joins[op.join];
		const std::string KT = jd.key64 ? "uint64_t" : "uint32_t";
		const std::string S = join_slot_type(jd);
		const std::string j = std::to_string(opi);
		for (int k = 0; k < op.npay; k++) {
			o << "    int64_t pay" << j << "_" << k << "[" << V << "];\n";
		}
		o << "    {\n";
		o << "      const " << S << "* __restrict__ jt" << j << " = " << Pptr(jd.table, "const " + S + "*") << ";\n";
		if (jd.direct) {
			o << "      const uint64_t bmask" << j << " = " << Pu(jd.direct_bmask) << ";\n";
		} else {
			/* staged build: the table was sized by the materialised count */
			o << "      const uint64_t bmask" << j << " = ((const unsigned long long*)" << Pptr(jd.words, "const void*")
			  << ")[1];\n";
		}
		o << "      constexpr int SPB" << j << " = vd::slots_per_bucket<" << S << ">();\n";
		o << "      uint64_t nb" << j << "[" << V << "]; int ns" << j << "[" << V << "]; uint64_t ng" << j << "[" << V << "]; "
		  << KT << " nk" << j << "[" << V << "]; bool np" << j << "[" << V << "];\n";
		o << "#pragma unroll\n      for (int v = 0; v < " << V << "; v++) {\n";
		std::string inrange = "act[v]";
		std::string packed = "0ull";
		for (size_t k = 0; k < op.keys.size(); k++) {
			const std::string kv = expr(op.keys[k], "v");
			const std::string lo = P((unsigned long long)(int64_t)jd.key_b[k].lo);
			const std::string span = Pu((unsigned long long)(int64_t)(jd.key_b[k].hi - jd.key_b[k].lo));
			inrange += " && (uint64_t)(" + kv + " - " + lo + ") <= " + span;
			packed += " | ((uint64_t)(" + kv + " - " + lo + ") << " + P((unsigned long long)jd.key_shift[k]) + ")";
		}
		o << "        const bool ok = " << inrange << ";\n";
		o << "        const uint64_t pk = " << packed << ";\n";
		o << "        nk" << j << "[v] = (" << KT << ")(pk + 1ull);\n";
		o << "        nb" << j << "[v] = (" << table_hash(op.keys, "pk", jd.key_bits, "v") << ") & bmask" << j << ";\n";
		o << "        ns" << j << "[v] = 0; ng" << j << "[v] = 0; np" << j << "[v] = ok;\n";
		o << "      }\n";
		o << "      for (;;) {\n";
		o << "        bool anyp = false;\n";
		o << "#pragma unroll\n        for (int v = 0; v < " << V << "; v++) { anyp = anyp || np" << j << "[v]; }\n";
		if (sink_block_collective()) {
			o << "        if (!vd::block_any(anyp)) { break; }\n";
		} else {
			o << "        if (!__any_sync(0xffffffffu, anyp)) { break; }\n";
		}
		o << "#pragma unroll\n        for (int v = 0; v < " << V << "; v++) {\n";
		o << "          uint64_t raw = 0;\n";
		o << "          act[v] = false;\n";
		o << "          while (np" << j << "[v]) {\n";
		/* duplicates cluster: a probe may walk the whole table, which always holds a free slot */
		o << "            if (++ng" << j << "[v] > (bmask" << j << " + 1ull) * SPB" << j << ") { atomicOr(err, VD_ERR_TABLE_FULL); np" << j
		  << "[v] = false; break; }\n";
		o << "            const " << S << "* sp = jt" << j << " + nb" << j << "[v] * SPB" << j << " + ns" << j << "[v];\n";
		o << "            const " << KT << " sk = vd::table_ld(&sp->key);\n";
		o << "            if (++ns" << j << "[v] == SPB" << j << ") { ns" << j << "[v] = 0; nb" << j << "[v] = (nb" << j
		  << "[v] + 1) & bmask" << j << "; }\n";
		o << "            if (sk == 0) { np" << j << "[v] = false; break; }\n";
		o << "            if (sk == nk" << j << "[v]) { act[v] = true; raw = (uint64_t)vd::table_ld(&sp->pay); break; }\n";
		o << "          }\n";
		emit_payload_unpack(op, jd, j, "raw");
		o << "        }\n";
		emit_rest(opi + 1);
		o << "      }\n";
		o << "    }\n";
	}

	/* one tile's work for the tile index `t`: loads (mode "ldg", "smem" or "pre" = the
	 * eager columns are already in x<c>), ops, sink */
	void emit_body(const std::string& mode) {
		o << "    {\n";
		o << "    const int64_t r0 = t * tile + (int64_t)threadIdx.x * " << V << ";\n";
		o << "    bool act[" << V << "];\n";
		o << "#pragma unroll\n    for (int v = 0; v < " << V << "; v++) { act[v] = r0 + v < n; }\n";
		if (mode != "pre") {
			emit_decl_cols(true, V);
			emit_load_cols(mode, "x", "r0");
		}
		if (compact_at < 0) {
			emit_rest(0);
			if (regs_acc) {
				/* block-uniform: every thread of the block runs the same tiles */
				o << "    if (++rtiles == " << regs_tiles << ") { rflush(); rtiles = 0; }\n";
			}
			o << "    }\n";
			return;
		}
		emit_ops(0, compact_at + 1);
		/* selection vector: the survivors' rows (and carried payloads) are appended to the
		 * block's pending buffer; the rest of the pipeline runs once at least a full pass of
		 * threads is pending, so every lane of the dependent gather/probe chain has a row */
		if (warp_compact()) {
			/* each warp appends its own survivors (ballot + rank) and flushes on its own */
			o << "    {\n      int wcnt = 0;\n";
			o << "#pragma unroll\n      for (int v = 0; v < " << V << "; v++) {\n";
			o << "        const unsigned m = __ballot_sync(0xffffffffu, act[v]);\n";
			o << "        if (act[v]) {\n";
			o << "          const int pos = cpend + wcnt + __popc(m & vd::lanemask_lt());\n";
			o << "          csel[pos] = r0 + v;\n";
			for (size_t k = 0; k < carried.size(); k++) {
				o << "          ccar" << k << "[pos] = pay" << carried[k].first << "_" << carried[k].second << "[v];\n";
			}
			o << "        }\n        wcnt += __popc(m);\n      }\n";
			o << "      cpend += wcnt;\n    }\n";
			o << "    __syncwarp();\n";
			o << "    if (cpend >= " << 32 * FV() << ") { cflush(); }\n";
			o << "    }\n";
			return;
		}
		o << "    const int nsel = vd::block_compact_rows<" << V << ">(act, r0, csel + cpend, cscan, csel_pos);\n";
		for (size_t k = 0; k < carried.size(); k++) {
			o << "#pragma unroll\n    for (int v = 0; v < " << V << "; v++) { if (act[v]) { ccar" << k
			  << "[cpend + csel_pos[v]] = pay" << carried[k].first << "_" << carried[k].second << "[v]; } }\n";
		}
		o << "    cpend += nsel;\n";
		o << "    vd::block_sync();\n";
		o << "    if (cpend >= " << T * FV() << ") { cflush(); }\n";
		o << "    }\n";
	}

	/* Shared-memory selection vector for compaction (declared once per kernel): room for a
	 * pass of threads still pending plus one more tile's survivors, and the flush that runs
	 * the pipeline's remaining ops and sink over the pending rows, one row per thread. */
	void emit_compaction_smem() {
		if (compact_at < 0) {
			return;
		}
		const bool wc = warp_compact();
		/* per warp (warp compaction) or per block: a flush's worth of rows plus one more tile */
		const int lanes = wc ? 32 : T;
		const int cap = lanes * FV() + lanes * V;
		/* row indices as 32 bits when every row of the table fits */
		const bool sel32 = p.rows <= (int64_t)UINT32_MAX;
		const std::string sel_t = sel32 ? "uint32_t" : "int64_t";
		/* the buffers live in dynamic shared memory after the sink's (before any tile ring) */
		const size_t copies = wc ? (size_t)(T / 32) : 1;
		size_t off = (smem_sink + 15) & ~(size_t)15;
		o << "  " << sel_t << "* const csel = (" << sel_t << "*)(vd_smem + " << off << ")"
		  << (wc ? " + (threadIdx.x >> 5) * " + std::to_string(cap) : std::string()) << ";\n";
		off += copies * cap * (sel32 ? 4 : 8);
		for (size_t k = 0; k < carried.size(); k++) {
			off = (off + 15) & ~(size_t)15;
			o << "  int64_t* const ccar" << k << " = (int64_t*)(vd_smem + " << off << ")"
			  << (wc ? " + (threadIdx.x >> 5) * " + std::to_string(cap) : std::string()) << ";\n";
			off += copies * cap * 8;
		}
		smem_sink = off;
		if (!wc) {
			o << "  __shared__ int cscan[33];\n";
			o << "  int csel_pos[" << V << "];\n";
		}
		o << "  int cpend = 0;\n";
		const int F = FV();
		const std::string lane_ix = wc ? "(int)vd::lane_id()" : "(int)threadIdx.x";
		o << "  auto cflush = [&]() {\n";
		o << "    for (int base = 0; base < cpend; base += " << lanes * F << ") {\n";
		o << "      bool act[" << F << "];\n      int64_t row[" << F << "];\n";
		o << "#pragma unroll\n      for (int v = 0; v < " << F << "; v++) {\n";
		o << "        const int ci = base + v * " << lanes << " + " << lane_ix << ";\n";
		o << "        act[v] = ci < cpend;\n";
		o << "        row[v] = act[v] ? (int64_t)csel[ci] : 0;\n";
		o << "      }\n";
		const int saveV = V;
		V = F;
		/* every column is gathered just before the first op (or the sink) that reads it, and
		 * only for rows still alive there: a row that fails a probe never touches the columns
		 * of the later ones */
		lazy_first_use.assign(p.cols.size(), INT32_MAX);
		for (size_t i = compact_at + 1; i < p.ops.size(); i++) {
			std::vector<bool> used(p.cols.size(), false);
			if (p.ops[i].pred) cols_of(p.ops[i].pred, used);
			for (auto& k : p.ops[i].keys) cols_of(k, used);
			for (size_t c = 0; c < p.cols.size(); c++) {
				if (used[c] && lazy_first_use[c] == INT32_MAX) {
					lazy_first_use[c] = (int)i;
				}
			}
		}
		{
			std::vector<bool> used(p.cols.size(), false);
			for (auto& e : sink_exprs()) cols_of(e, used);
			for (size_t c = 0; c < p.cols.size(); c++) {
				if (used[c] && lazy_first_use[c] == INT32_MAX) {
					lazy_first_use[c] = (int)p.ops.size();
				}
			}
		}
		for (size_t c = 0; c < p.cols.size(); c++) {
			if (lazy_first_use[c] != INT32_MAX) {
				o << "      " << ctype(p.cols[c].type) << " x" << c << "[" << F << "] = {0};\n";
			}
		}
		for (size_t k = 0; k < carried.size(); k++) {
			const std::string pv = "pay" + std::to_string(carried[k].first) + "_" + std::to_string(carried[k].second);
			o << "      int64_t " << pv << "[" << F << "];\n";
			o << "#pragma unroll\n      for (int v = 0; v < " << F << "; v++) { " << pv << "[v] = act[v] ? ccar" << k << "[base + v * "
			  << lanes << " + " << lane_ix << "] : 0; }\n";
		}
		lazy_rows = true;
		emit_rest(compact_at + 1);
		lazy_rows = false;
		V = saveV;
		o << "    }\n";
		o << (wc ? "    __syncwarp();\n" : "    vd::block_sync();\n");
		o << "    cpend = 0;\n";
		o << "  };\n";
	}

	/* payload outputs of a probe from the packed payload `raw` */
	void emit_payload_unpack(const Op& op, const JoinDesc& jd, const std::string& j, const std::string& raw) {
		for (int k = 0; k < op.npay; k++) {
			const int bits = (k + 1 < op.npay ? jd.pay_shift[k + 1] : jd.pay_bits) - jd.pay_shift[k];
			const unsigned long long mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1ull);
			o << "        pay" << j << "_" << k << "[v] = " << P((unsigned long long)(int64_t)jd.pay_b[k].lo)
			  << " + (int64_t)(((uint64_t)" << raw << " >> " << P((unsigned long long)jd.pay_shift[k]) << ") & "
			  << Pu(mask) << ");\n";
		}
	}

	/* probe of a dense join table: the packed key indexes the table directly */
	void gen_probe_dense(const Op& op, const JoinDesc& jd, const std::string& j) {
		const int eb = jd.dense_entry_bytes();
		const std::string ET = eb == 8 ? "unsigned long long" : "unsigned";
		o << "    {\n";
		o << "      const " << ET << "* __restrict__ jd" << j << " = " << Pptr(jd.table, "const " + ET + "*") << ";\n";
		o << "#pragma unroll\n      for (int v = 0; v < " << V << "; v++) {\n";
		std::string inrange = "act[v]";
		std::string packed = "0ull";
		for (size_t k = 0; k < op.keys.size(); k++) {
			const std::string kv = expr(op.keys[k], "v");
			const std::string lo = P((unsigned long long)(int64_t)jd.key_b[k].lo);
			const std::string span = Pu((unsigned long long)(int64_t)(jd.key_b[k].hi - jd.key_b[k].lo));
			inrange += " && (uint64_t)(" + kv + " - " + lo + ") <= " + span;
			packed += " | ((uint64_t)(" + kv + " - " + lo + ") << " + P((unsigned long long)jd.key_shift[k]) + ")";
		}
		o << "        const bool ok = " << inrange << ";\n";
		o << "        const uint64_t pk = " << packed << ";\n";
		if (eb == 0) {
			o << "        act[v] = ok && vd::dense_test(jd" << j << ", pk);\n";
		} else {
			o << "        const " << ET << " e = ok ? vd::table_ld(&jd" << j << "[pk]) : (" << ET << ")0;\n";
			o << "        act[v] = e != 0;\n";
			o << "        const uint64_t raw = e != 0 ? (uint64_t)e - 1ull : 0ull;\n";
			emit_payload_unpack(op, jd, j, "raw");
		}
		o << "      }\n";
		o << "    }\n";
	}

	void gen_probe(int opi, const Op& op) {
		JoinDesc& jd = plan.joins[op.join];
		const std::string KT = jd.key64 ? "uint64_t" : "uint32_t";
		const std::string PT = jd.pay64 ? "uint64_t" : "uint32_t";
		const std::string S = join_slot_type(jd);
		const std::string j = std::to_string(opi);
		for (int k = 0; k < op.npay; k++) {
			o << "    int64_t pay" << j << "_" << k << "[" << V << "];\n";
		}
		if (jd.dense) {
			gen_probe_dense(op, jd, j);
			return;
		}
		o << "    {\n";
		o << "      const " << S << "* __restrict__ jt = " << Pptr(jd.table, "const " + S + "*") << ";\n";
		if (jd.direct) {
			o << "      const uint64_t bmask = " << Pu(jd.direct_bmask) << ";\n";
		} else {
			o << "      const uint64_t bmask = ((const unsigned long long*)" << Pptr(jd.words, "const void*") << ")[1];\n";
		}
		if (fl.probe_lanes > 1) {
			gen_probe_coop(op, jd, j);
			return;
		}
		o << "      int st[" << V << "]; uint64_t bk[" << V << "]; " << KT << " key[" << V << "]; " << PT
		  << " raw[" << V << "];\n";
		o << "#pragma unroll\n      for (int v = 0; v < " << V << "; v++) {\n";
		std::string inrange = "act[v]";
		std::string packed = "0ull";
		for (size_t k = 0; k < op.keys.size(); k++) {
			const std::string kv = expr(op.keys[k], "v");
			const std::string lo = P((unsigned long long)(int64_t)jd.key_b[k].lo);
			const std::string span = Pu((unsigned long long)(int64_t)(jd.key_b[k].hi - jd.key_b[k].lo));
			/* keys outside the build side's domain cannot match (and must not alias) */
			inrange += " && (uint64_t)(" + kv + " - " + lo + ") <= " + span;
			packed += " | ((uint64_t)(" + kv + " - " + lo + ") << " + P((unsigned long long)jd.key_shift[k]) + ")";
		}
		o << "        const bool ok = " << inrange << ";\n";
		o << "        const uint64_t pk = " << packed << ";\n";
		o << "        key[v] = (" << KT << ")(pk + 1ull);\n";
		o << "        bk[v] = " << table_hash(op.keys, "pk", jd.key_bits, "v") << " & bmask;\n";
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
		emit_payload_unpack(op, jd, j, "raw[v]");
		o << "      }\n";
		o << "    }\n";
	}

	/*
	 * Warp-cooperative probe (flavor probe=G): the G lanes of a lane group take the group's
	 * keys one after another; for each key every lane reads a different bucket of its probe
	 * sequence (b, b+1, ..., b+G-1), and a ballot over the group finds the earliest bucket that
	 * holds the key (a match) or an empty slot (no match) -- linear probing never places a key
	 * past an empty slot of its sequence.  Long probe sequences then cost one round trip per
	 * G buckets instead of one per bucket; all lanes of a group stay converged.  Emitted inside
	 * gen_probe's block after the table pointer and bucket mask (jt, bmask).
	 */
	void gen_probe_coop(const Op& op, const JoinDesc& jd, const std::string& j) {
		const std::string KT = jd.key64 ? "uint64_t" : "uint32_t";
		const std::string PT = jd.pay64 ? "uint64_t" : "uint32_t";
		const int G = fl.probe_lanes;
		o << "      const unsigned cl = vd::lane_id() & " << (G - 1) << "u, cbase = vd::lane_id() & ~" << (G - 1) << "u;\n";
		o << "      const unsigned cmask = " << (G == 32 ? std::string("0xffffffffu") : "(" + std::to_string((1u << G) - 1u) + "u << cbase)")
		  << ";\n";
		o << "      bool cok[" << V << "]; uint64_t bk[" << V << "]; " << KT << " key[" << V << "];\n";
		o << "#pragma unroll\n      for (int v = 0; v < " << V << "; v++) {\n";
		std::string inrange = "act[v]";
		std::string packed = "0ull";
		for (size_t k = 0; k < op.keys.size(); k++) {
			const std::string kv = expr(op.keys[k], "v");
			const std::string lo = P((unsigned long long)(int64_t)jd.key_b[k].lo);
			const std::string span = Pu((unsigned long long)(int64_t)(jd.key_b[k].hi - jd.key_b[k].lo));
			inrange += " && (uint64_t)(" + kv + " - " + lo + ") <= " + span;
			packed += " | ((uint64_t)(" + kv + " - " + lo + ") << " + P((unsigned long long)jd.key_shift[k]) + ")";
		}
		o << "        cok[v] = " << inrange << ";\n";
		o << "        const uint64_t pk = " << packed << ";\n";
		o << "        key[v] = (" << KT << ")(pk + 1ull);\n";
		o << "        bk[v] = " << table_hash(op.keys, "pk", jd.key_bits, "v") << " & bmask;\n";
		o << "      }\n";
		o << "#pragma unroll\n      for (int v = 0; v < " << V << "; v++) {\n";
		o << "        int mine = 0; " << PT << " myraw = 0;\n";
		o << "        for (unsigned src = 0; src < " << G << "u; src++) {\n";
		o << "          const bool ok = __shfl_sync(cmask, (unsigned)cok[v], cbase + src) != 0u;\n";
		o << "          const " << KT << " k = __shfl_sync(cmask, key[v], cbase + src);\n";
		o << "          uint64_t b = __shfl_sync(cmask, (unsigned long long)bk[v], cbase + src);\n";
		o << "          int res = 0; " << PT << " r = 0;\n";
		o << "          if (ok) {\n";
		o << "            int step = 0;\n";
		o << "            for (; step < VD_MAX_PROBES; step += " << G << ") {\n";
		o << "              " << PT << " rr = 0;\n";
		o << "              const int s = vd::join_probe_bucket(jt, (b + cl) & bmask, k, rr);\n";
		o << "              const unsigned hit = __ballot_sync(cmask, s == 1) & cmask;\n";
		o << "              const unsigned fin = (__ballot_sync(cmask, s == 0) & cmask) | hit;\n";
		o << "              if (fin) {\n";
		o << "                const int first = __ffs(fin) - 1;\n";
		o << "                r = __shfl_sync(cmask, rr, first);\n";
		o << "                res = (hit >> first) & 1u;\n";
		o << "                break;\n";
		o << "              }\n";
		o << "              b += " << G << ";\n";
		o << "            }\n";
		o << "            if (step >= VD_MAX_PROBES && cl == 0) { atomicOr(err, VD_ERR_TABLE_FULL); }\n";
		o << "          }\n";
		o << "          if (cl == src) { mine = res; myraw = r; }\n";
		o << "        }\n";
		o << "        act[v] = mine == 1;\n";
		emit_payload_unpack(op, jd, j, "myraw");
		o << "      }\n";
		o << "    }\n";
	}

	/* ------------------------------------------------------------ sinks ------------ */

	void sink_prologue() {
		Sink& s = p.sink;
		switch (s.kind) {
		case Sink::AggGlobal:
			o << "  int64_t acc[" << A() << "];\n";
			o << "#pragma unroll\n  for (int a = 0; a < " << A() << "; a++) { acc[a] = 0; }\n";
			break;
		case Sink::AggDense: {
			const int64_t D = (int64_t)s.domain;
			const int64_t warps = T / 32;
			const int64_t slot_bytes = D * A() * 8;
			const int64_t cap = std::min<int64_t>(96 * 1024, fl.sink_smem);
			if (fl.lowcard == "atomic") {
				replicas = slot_bytes * warps <= cap ? (int)warps : 1;
			} else if (fl.lowcard == "redux") {
				/* one copy of the slots per warp (or per group of warps) within 64 KiB: the
				 * group leaders of a warp then update their own copy */
				replicas = (int)std::max<int64_t>(1, std::min<int64_t>(warps, std::min<int64_t>(64 * 1024, cap) /
					std::max<int64_t>(slot_bytes, 1)));
			} else {
				replicas = 1;
			}
			dense_in_smem = slot_bytes * replicas <= cap;
			if (!dense_in_smem) {
				replicas = 1;
			}
			/* every warp owns its copy: leaders (distinct slots within a warp) add without atomics */
			leader_plain = fl.lowcard == "redux" && dense_in_smem && replicas == warps;
			if (dense_in_smem) {
				smem_sink = (size_t)(D * A() * 8 * replicas);
				o << "  unsigned long long* const sacc0 = (unsigned long long*)vd_smem;\n";
				o << "  for (int64_t i = threadIdx.x; i < " << P((unsigned long long)(D * A() * replicas))
				  << "; i += blockDim.x) { sacc0[i] = 0ull; }\n";
				o << "  vd::block_sync();\n";
				if (replicas > 1) {
					o << "  unsigned long long* const sacc = sacc0 + ((threadIdx.x >> 5) % " << replicas << ") * "
					  << P((unsigned long long)(D * A())) << ";\n";
				} else {
					o << "  unsigned long long* const sacc = sacc0;\n";
				}
			} else {
				o << "  unsigned long long* const sacc = " << Pptr(st.sink_dev, "unsigned long long*") << ";\n";
			}
			/* per-thread private accumulators for up to kGmax slots seen by the block */
			const size_t priv_bytes = (size_t)kGmax * A() * T * 8;
			const size_t dict_bytes = ((size_t)D * 4 + 4 * (kGmax + 1) + 15) & ~(size_t)15;
			private_acc = fl.lowcard == "private" && dense_in_smem && replicas == 1 &&
				smem_sink + priv_bytes + dict_bytes <= 160 * 1024;
			if (private_acc) {
				const size_t priv_off = (smem_sink + 15) & ~(size_t)15;
				const size_t dict_off = priv_off + priv_bytes;
				smem_sink = dict_off + dict_bytes;
				o << "  int64_t* const priv = (int64_t*)(vd_smem + " << priv_off << ");\n";
				o << "  int* const pdict = (int*)(vd_smem + " << dict_off << ");\n";
				o << "  int* const pcodes = pdict + " << P((unsigned long long)D) << ";\n";
				o << "  int* const pncodes = pcodes + " << kGmax << ";\n";
				o << "  for (int64_t i = threadIdx.x; i < " << P((unsigned long long)D)
				  << "; i += blockDim.x) { pdict[i] = -1; }\n";
				o << "  if (threadIdx.x == 0) { *pncodes = 0; }\n";
				o << "#pragma unroll\n  for (int i = 0; i < " << kGmax * A() << "; i++) { priv[i * " << T
				  << " + threadIdx.x] = 0; }\n";
				o << "  vd::block_sync();\n";
			}
			/* per-thread packed accumulator words (registers for regs, a shared-memory column
			 * per thread for packed) for up to kGmax slots (codes of the block's dictionary),
			 * summed over regs_tiles tiles, then folded per warp by redux.sync into the block's
			 * slot array */
			regs_smem = fl.lowcard == "packed";
			regs_acc = (fl.lowcard == "regs" || regs_smem) && dense_in_smem && replicas == 1 && !item && compact_at < 0 &&
				A() <= 32 &&
				!has_join_n() && plan_regs();
			if (regs_acc) {
				const size_t dict_bytes = ((size_t)D * 4 + 4 * (kGmax + 1) + 15) & ~(size_t)15;
				const size_t dict_off = (smem_sink + 15) & ~(size_t)15;
				smem_sink = dict_off + dict_bytes;
				const int RW = regs_words;
				o << "  int* const pdict = (int*)(vd_smem + " << dict_off << ");\n";
				o << "  int* const pcodes = pdict + " << P((unsigned long long)D) << ";\n";
				o << "  int* const pncodes = pcodes + " << kGmax << ";\n";
				o << "  for (int64_t i = threadIdx.x; i < " << P((unsigned long long)D)
				  << "; i += blockDim.x) { pdict[i] = -1; }\n";
				o << "  if (threadIdx.x == 0) { *pncodes = 0; }\n";
				if (regs_smem) {
					/* word j of code k of this thread at pacc[(k * RW + j) * T + thread] */
					const size_t pacc_off = (smem_sink + 15) & ~(size_t)15;
					smem_sink = pacc_off + (size_t)kGmax * RW * T * 8;
					o << "  uint64_t* const pacc = (uint64_t*)(vd_smem + " << pacc_off << ") + threadIdx.x;\n";
					o << "#define racc(k, j) pacc[((k) * " << RW << " + (j)) * " << T << "]\n";
				} else {
					o << "  uint64_t racc_r[" << kGmax << "][" << RW << "];\n";
					o << "#define racc(k, j) racc_r[k][j]\n";
				}
				o << "#pragma unroll\n  for (int k = 0; k < " << kGmax << "; k++) {\n";
				o << "#pragma unroll\n    for (int j = 0; j < " << RW << "; j++) { racc(k, j) = 0ull; }\n  }\n";
				o << "  int rtiles = 0;\n";
				o << "  vd::block_sync();\n";
				/* warp-collective: every lane of the warp calls it at the same point */
				const int cw = rg_word[s.count_idx];
				o << "  auto rflush = [&]() {\n";
				o << "    __threadfence_block();\n";
				o << "#pragma unroll\n    for (int k = 0; k < " << kGmax << "; k++) {\n";
				o << "      if (__any_sync(0xffffffffu, racc(k, " << cw << ") != 0ull)) {\n";
				o << "        const int64_t sl = (int64_t)((volatile int*)pcodes)[k];\n";
				o << "        uint64_t rw[" << RW << "];\n";
				o << "#pragma unroll\n        for (int j = 0; j < " << RW << "; j++) { rw[j] = racc(k, j); }\n";
				auto field = [&](int a) {
					const unsigned long long mask = rg_bits[a] >= 64 ? ~0ull : ((1ull << rg_bits[a]) - 1ull);
					return "vd::group_sum_u<" + std::to_string(rg_bits[a]) + ">(0xffffffffu, (rw[" +
						std::to_string(rg_word[a]) + "] >> " + std::to_string(rg_shift[a]) + ") & " +
						std::to_string(mask) + "ull)";
				};
				o << "        const uint64_t cnt = " << field(s.count_idx) << ";\n";
				o << "        uint64_t mine = 0ull;\n";
				for (int a = 0; a < A(); a++) {
					if (a == s.count_idx) {
						o << "        if (vd::lane_id() == " << a << "u) { mine = cnt; }\n";
					} else if (s.aggs[a].count) {
						o << "        if (vd::lane_id() == " << a << "u) { mine = " << field(a) << "; }\n";
					} else {
						o << "        { const uint64_t sa = " << field(a) << " + (uint64_t)"
						  << P((unsigned long long)(int64_t)s.aggs[a].arg->b.lo) << " * cnt;\n";
						o << "          if (vd::lane_id() == " << a << "u) { mine = sa; } }\n";
					}
				}
				o << "        if (vd::lane_id() < " << A() << "u && mine != 0ull) { atomicAdd(&sacc[sl * " << A()
				  << " + vd::lane_id()], (unsigned long long)mine); }\n";
				o << "#pragma unroll\n        for (int j = 0; j < " << RW << "; j++) { racc(k, j) = 0ull; }\n";
				o << "      }\n    }\n  };\n";
			}
			break;
		}
		case Sink::AggHash: {
			if (part()) {
				part_prologue();
				break;
			}
			const std::string K = gkey_type();
			const int W = s.nwords;
			if (gdirect()) {
				o << "  unsigned long long* const gacc = " << Pptr(st.sink_acc, "unsigned long long*") << ";\n";
			} else {
				o << "  " << K << "* const gkeys = " << Pptr(st.sink_dev, K + "*") << ";\n";
				o << "  unsigned long long* const gacc = " << Pptr(st.sink_acc, "unsigned long long*") << ";\n";
				o << "  const uint64_t gbmask = " << Pu((unsigned long long)(st.sink_cap / (32 / gkey_bytes()) - 1)) << ";\n";
			}
			if (gcache()) {
				const int S = (int)pow2_at_least(std::max(32, fl.cache_slots));
				const size_t kbytes = ((size_t)S * gkey_bytes() + 15) & ~(size_t)15;
				smem_sink = kbytes + (size_t)S * W * 8;
				o << "  " << K << "* const ckeys = (" << K << "*)vd_smem;\n";
				o << "  unsigned long long* const cacc = (unsigned long long*)(vd_smem + " << kbytes << ");\n";
				o << "  for (int i = threadIdx.x; i < " << S << "; i += blockDim.x) { ckeys[i] = 0; }\n";
				o << "  for (int i = threadIdx.x; i < " << S * W << "; i += blockDim.x) { cacc[i] = 0ull; }\n";
				o << "  vd::block_sync();\n";
				cache_slots = S;
			}
			break;
		}
		case Sink::JoinBuild: {
			JoinDesc& jd = plan.joins[s.join];
			const std::string S = join_slot_type(jd);
			if (jd.dense) {
				const std::string ET = jd.dense_entry_bytes() == 8 ? "unsigned long long" : "unsigned";
				o << "  " << ET << "* const jdt = " << Pptr(jd.table, ET + "*") << ";\n";
			} else if (jd.direct) {
				o << "  " << S << "* const jt = " << Pptr(jd.table, S + "*") << ";\n";
				o << "  const uint64_t bmask = " << Pu(jd.direct_bmask) << ";\n";
			} else {
				o << "  __shared__ unsigned long long app[33];\n";
				o << "  unsigned long long* const words = " << Pptr(jd.words, "unsigned long long*") << ";\n";
				o << "  " << (jd.key64 ? "uint64_t" : "uint32_t") << "* const skeys = "
				  << Pptr(jd.stage_keys, jd.key64 ? "uint64_t*" : "uint32_t*") << ";\n";
				o << "  " << (jd.pay64 ? "uint64_t" : "uint32_t") << "* const spay = "
				  << Pptr(jd.stage_pay, jd.pay64 ? "uint64_t*" : "uint32_t*") << ";\n";
				o << "  uint64_t* const shash = " << Pptr(st.stage_hash, "uint64_t*") << ";\n";
			}
			break;
		}
		case Sink::Emit:
			o << "  __shared__ unsigned long long app[33];\n";
			o << "  int64_t* const out = " << Pptr(qs.out, "int64_t*") << ";\n";
			o << "  const int64_t ocap = " << P((unsigned long long)qs.out_cap) << ";\n";
			o << "  unsigned long long* const ocount = " << Pptr(qs.out_count, "unsigned long long*") << ";\n";
			break;
		}
	}

	std::string packed_key(const std::vector<BExprP>& keys, const std::vector<Bounds>& b, const std::vector<int>& shift,
		const std::string& v) {
		std::string pk = "0ull";
		for (size_t k = 0; k < keys.size(); k++) {
			pk += " | ((uint64_t)(" + expr(keys[k], v) + " - " + P((unsigned long long)(int64_t)b[k].lo) + ") << " +
				P((unsigned long long)shift[k]) + ")";
		}
		return pk;
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
			/* a slot array in shared memory has fewer than 2^31 slots: 32-bit index arithmetic */
			const bool slot32 = dense_in_smem;
			for (size_t k = 0; k < s.keys.size(); k++) {
				if (slot32) {
					slot += " + (int)(" + expr(s.keys[k], "v") + " - " + P((unsigned long long)(int64_t)s.keys[k]->b.lo) +
						") * (int)" + P((unsigned long long)s.key_radix[k]);
				} else {
					slot += " + (" + expr(s.keys[k], "v") + " - " + P((unsigned long long)(int64_t)s.keys[k]->b.lo) +
						") * " + P((unsigned long long)s.key_radix[k]);
				}
			}
			o << "      const int64_t slot = act[v] ? (int64_t)(" << slot << ") : 0;\n";
			o << "      " << agg_vals("v") << "\n";
			if (regs_acc) {
				o << "      const int code = act[v] ? vd::dict_code(pdict, pcodes, pncodes, slot, " << kGmax << ") : -2;\n";
				o << "      if (code == -1) {\n";
				o << "#pragma unroll\n        for (int a = 0; a < " << A() << "; a++) { "
				  << "atomicAdd(&sacc[slot * " << A() << " + a], (unsigned long long)vals[a]); }\n";
				o << "      }\n";
				for (int j = 0; j < regs_words; j++) {
					o << "      const uint64_t rw" << j << " = 0ull";
					for (int a = 0; a < A(); a++) {
						if (rg_word[a] != j) {
							continue;
						}
						if (s.aggs[a].count) {
							o << " + (1ull << " << rg_shift[a] << ")";
						} else {
							o << " + (((uint64_t)vals[" << a << "] - (uint64_t)" << P((unsigned long long)(int64_t)s.aggs[a].arg->b.lo)
							  << ") << " << rg_shift[a] << ")";
						}
					}
					o << ";\n";
				}
				if (regs_smem) {
					o << "      if (code >= 0) {\n";
					for (int j = 0; j < regs_words; j++) {
						o << "        racc(code, " << j << ") += rw" << j << ";\n";
					}
					o << "      }\n    }\n";
				} else {
					o << "#pragma unroll\n      for (int k = 0; k < " << kGmax << "; k++) {\n";
					for (int j = 0; j < regs_words; j++) {
						o << "        racc(k, " << j << ") += code == k ? rw" << j << " : 0ull;\n";
					}
					o << "      }\n    }\n";
				}
				break;
			}
			if (private_acc) {
				o << "      if (act[v]) {\n";
				o << "        const int code = vd::dict_code(pdict, pcodes, pncodes, slot, " << kGmax << ");\n";
				o << "        if (code >= 0) {\n";
				o << "#pragma unroll\n          for (int a = 0; a < " << A() << "; a++) { priv[(code * " << A() << " + a) * "
				  << T << " + threadIdx.x] += vals[a]; }\n";
				o << "        } else {\n";
				o << "#pragma unroll\n          for (int a = 0; a < " << A() << "; a++) { atomicAdd(&sacc[slot * " << A() << " + a], (unsigned long long)vals[a]); }\n";
				o << "        }\n      }\n    }\n";
				break;
			}
			if (fl.lowcard == "atomic") {
				o << "      if (act[v]) {\n";
			} else if (fl.lowcard == "redux") {
				emit_group_reduce("act[v] ? (unsigned)slot : 0xffffffffu");
				o << "      if (lead) {\n";
			} else {
				o << "      if (vd::warp_combine<" << A() << ">((uint64_t)slot, act[v], vals)) {\n";
			}
			if (leader_plain) {
				o << "#pragma unroll\n        for (int a = 0; a < " << A() << "; a++) { sacc[slot * " << A()
				  << " + a] += (unsigned long long)vals[a]; }\n";
			} else {
				o << "#pragma unroll\n        for (int a = 0; a < " << A() << "; a++) { atomicAdd(&sacc[slot * " << A() << " + a], (unsigned long long)vals[a]); }\n";
			}
			o << "      }\n    }\n";
			break;
		}
		case Sink::AggHash: {
			std::vector<Bounds> kb;
			for (auto& k : s.keys) {
				kb.push_back(k->b);
			}
			if (part()) {
				part_row(kb);
				break;
			}
			const std::string K = gkey_type();
			const int W = s.nwords;
			if (gdirect() && !gcache()) {
				/* direct table: each group leader adds its warp's pre-sums at slot = packed key */
				o << "#pragma unroll\n    for (int v = 0; v < " << V << "; v++) {\n";
				o << "      const uint64_t pk = act[v] ? (" << packed_key(s.keys, kb, s.key_shift, "v") << ") : 0ull;\n";
				emit_packed_words(p.sink.key_bits <= 31 ? "act[v] ? (unsigned)pk : 0xffffffffu" : "act[v] ? (unsigned long long)pk : ~0ull", "v");
				o << "      if (lead) { vd::gt_add<" << W << ">(gacc, (int64_t)pk, w); }\n";
				o << "    }\n";
				break;
			}
			if (!gcache()) {
				/* three phases so each thread keeps V bucket loads in flight: warp pre-sums of
				 * every row, then the first bucket of every leader's probe, then the inserts
				 * and atomics */
				o << "    uint64_t hk[" << V << "]; " << K << " kk[" << V << "]; bool ldr[" << V << "]; uint64_t ww[" << V
				  << "][" << W << "];\n";
				o << "#pragma unroll\n    for (int v = 0; v < " << V << "; v++) {\n";
				o << "      const uint64_t pk = act[v] ? (" << packed_key(s.keys, kb, s.key_shift, "v") << ") : 0ull;\n";
				emit_packed_words(p.sink.key_bits <= 31 ? "act[v] ? (unsigned)pk : 0xffffffffu" : "act[v] ? (unsigned long long)pk : ~0ull", "v");
				o << "      ldr[v] = lead;\n      kk[v] = (" << K << ")(pk + 1ull);\n";
				o << "      hk[v] = " << table_hash(s.keys, "pk", s.key_bits, "v") << ";\n";
				o << "#pragma unroll\n      for (int a = 0; a < " << W << "; a++) { ww[v][a] = w[a]; }\n";
				o << "    }\n";
				o << "    uint4 bq0[" << V << "], bq1[" << V << "];\n";
				o << "#pragma unroll\n    for (int v = 0; v < " << V << "; v++) {\n";
				o << "      if (ldr[v]) {\n";
				o << "        const uint4* bp = reinterpret_cast<const uint4*>(gkeys + (hk[v] & gbmask) * "
				  << 32 / gkey_bytes() << ");\n";
				o << "        bq0[v] = __ldcg(bp);\n        bq1[v] = __ldcg(bp + 1);\n      }\n    }\n";
				o << "#pragma unroll\n    for (int v = 0; v < " << V << "; v++) {\n";
				o << "      if (ldr[v]) {\n";
				o << "        const int64_t slot = vd::gt_find_or_insert_pre<" << K << ">(gkeys, gbmask, hk[v], kk[v], bq0[v], bq1[v], err);\n";
				o << "        if (slot >= 0) { vd::gt_add<" << W << ">(gacc, slot, ww[v]); }\n";
				o << "      }\n    }\n";
				break;
			}
			o << "#pragma unroll\n    for (int v = 0; v < " << V << "; v++) {\n";
			o << "      const uint64_t pk = act[v] ? (" << packed_key(s.keys, kb, s.key_shift, "v") << ") : 0ull;\n";
			emit_packed_words(p.sink.key_bits <= 31 ? "act[v] ? (unsigned)pk : 0xffffffffu" : "act[v] ? (unsigned long long)pk : ~0ull", "v");
			o << "      if (lead) {\n";
			o << "        const uint64_t h = " << table_hash(s.keys, "pk", s.key_bits, "v") << ";\n";
			o << "        const " << K << " key = (" << K << ")(pk + 1ull);\n";
			if (gcache()) {
				o << "        if (!vd::gt_cache_add<" << K << ", " << W << ">(ckeys, cacc, " << cache_slots << ", h, key, w)) {\n";
				if (gdirect()) {
					o << "          vd::gt_add<" << W << ">(gacc, (int64_t)pk, w);\n";
				} else {
					o << "          const int64_t slot = vd::gt_find_or_insert<" << K << ">(gkeys, gbmask, h, key, err);\n";
					o << "          if (slot >= 0) { vd::gt_add<" << W << ">(gacc, slot, w); }\n";
				}
				o << "        }\n";
			} else {
				o << "        const int64_t slot = vd::gt_find_or_insert<" << K << ">(gkeys, gbmask, h, key, err);\n";
				o << "        if (slot >= 0) { vd::gt_add<" << W << ">(gacc, slot, w); }\n";
			}
			o << "      }\n    }\n";
			break;
		}
		case Sink::JoinBuild: {
			JoinDesc& jd = plan.joins[s.join];
			const std::string KT = jd.key64 ? "uint64_t" : "uint32_t";
			const std::string PT = jd.pay64 ? "uint64_t" : "uint32_t";
			o << "#pragma unroll\n    for (int v = 0; v < " << V << "; v++) {\n";
			const std::string pk = packed_key(s.keys, jd.key_b, jd.key_shift, "v");
			const std::string pp = s.pay.empty() ? std::string("0ull") : packed_key(s.pay, jd.pay_b, jd.pay_shift, "v");
			if (jd.dense) {
				o << "      if (act[v]) {\n";
				o << "        const uint64_t pkb = " << pk << ";\n";
				if (jd.dense_entry_bytes() == 0) {
					o << "        vd::dense_set(jdt, pkb);\n";
				} else {
					const std::string ET = jd.dense_entry_bytes() == 8 ? "unsigned long long" : "unsigned";
					o << "        atomicCAS(&jdt[pkb], (" << ET << ")0, (" << ET << ")(" << pp << " + 1ull));\n";
				}
				o << "      }\n    }\n";
			} else if (jd.direct) {
				o << "      if (act[v]) {\n";
				o << "        const uint64_t pkb = " << pk << ";\n";
				o << "        vd::join_insert(jt, bmask, " << table_hash(s.keys, "pkb", jd.key_bits, "v") << ", (" << KT
				  << ")(pkb + 1ull), (" << PT << ")(" << pp << "), err" << (jd.join01 ? "" : ", bmask + 1ull") << ");\n";
				o << "      }\n    }\n";
			} else {
				o << "      const int64_t pos = vd::block_append(&words[0], act[v], app);\n";
				o << "      if (act[v]) {\n";
				o << "        const uint64_t pkb = " << pk << ";\n        skeys[pos] = (" << KT << ")(pkb + 1ull);\n";
				o << "        spay[pos] = (" << PT << ")(" << pp << ");\n";
				o << "        shash[pos] = " << table_hash(s.keys, "pkb", jd.key_bits, "v") << ";\n";
				o << "      }\n    }\n";
			}
			break;
		}
		case Sink::Emit: {
			o << "#pragma unroll\n    for (int v = 0; v < " << V << "; v++) {\n";
			o << "      const int64_t pos = vd::block_append(ocount, act[v], app);\n";
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

	/* the last CTA writes the result rows of a global or dense aggregation */
	void publish_slots(const std::string& g, int64_t nslots_val) {
		Sink& s = p.sink;
		o << "  __shared__ int last_flag;\n";
		o << "  if (vd::last_block_done(" << Pptr(st.done, "unsigned long long*") << ", " << blocks_total()
		  << ", &last_flag)) {\n";
		o << "    int64_t* const out = " << Pptr(qs.out, "int64_t*") << ";\n";
		o << "    const int64_t ocap = " << P((unsigned long long)qs.out_cap) << ";\n";
		o << "    unsigned long long* const ocount = " << Pptr(qs.out_count, "unsigned long long*") << ";\n";
		o << "    const int64_t nslots = " << P((unsigned long long)nslots_val) << ";\n";
		o << "    for (int64_t base = (threadIdx.x & ~31); base < nslots; base += blockDim.x) {\n";
		o << "      const int64_t i = base + (threadIdx.x & 31);\n";
		o << "      const bool take = i < nslots && (int64_t)__ldcg(&" << g << "[i * " << A() << " + " << s.count_idx
		  << "]) > 0;\n";
		o << "      const int64_t pos = vd::warp_append(ocount, take);\n";
		o << "      if (take && pos < ocap) {\n";
		int col = 0;
		for (size_t k = 0; k < s.keys.size(); k++, col++) {
			const int64_t range = (int64_t)(s.keys[k]->b.hi - s.keys[k]->b.lo + 1);
			o << "        out[" << col << " * ocap + pos] = " << P((unsigned long long)(int64_t)s.keys[k]->b.lo)
			  << " + (i / " << P((unsigned long long)s.key_radix[k]) << ") % " << P((unsigned long long)range) << ";\n";
		}
		for (int a = 0; a < A(); a++) {
			if (!s.aggs[a].visible) {
				continue;
			}
			o << "        out[" << col << " * ocap + pos] = (int64_t)__ldcg(&" << g << "[i * " << A() << " + " << a
			  << "]);\n";
			col++;
		}
		o << "      }\n    }\n  }\n";
	}

	/* ------------------------------------------------------- partitioned aggregation ---- */

	/* per-run words of a partitioned group-by (PartPlan::ctl): item counter, partial-run
	 * cursor, histogram done counter, then P record totals, P partition starts, P scatter
	 * cursors (64-bit) and P split-item done counters (32-bit) */
	std::string part_ctl_decl() {
		const PartPlan& pp = st.part;
		const int NP = pp.P;
		std::ostringstream d;
		d << "  unsigned long long* const pctl = " << Pptr(pp.ctl, "unsigned long long*") << ";\n";
		d << "  unsigned long long* const ptot = pctl + 4;\n";
		d << "  unsigned long long* const pstart = pctl + 4 + " << NP << ";\n";
		d << "  unsigned long long* const pcur = pctl + 4 + " << 2 * NP << ";\n";
		d << "  unsigned* const pdone = (unsigned*)(pctl + 4 + " << 3 * NP << ");\n";
		d << "  (void)ptot; (void)pstart; (void)pcur; (void)pdone;\n";
		return d.str();
	}

	/* partition of packed key pk: the top log2 P bits of its hash (the slot in a partition's
	 * table takes the low bits) */
	std::string part_of(const std::string& pk) {
		return "((uint32_t)vd::mix_hash32((uint32_t)(" + pk + ")) >> " + std::to_string(32 - st.part.log2P) + ")";
	}

	/* pass 0 (histogram) and pass 1 (scatter) state.  Both passes run the same grid over the
	 * same tiles, so CTA b of pass 1 emits exactly the records CTA b of pass 0 counted.  Pass 0
	 * counts each partition's rows in shared memory and writes its row of the count matrix;
	 * the last CTA turns the totals into partition starts.  Pass 1 reserves, for each
	 * partition, its CTA's run with one atomic on the partition's cursor, then writes each
	 * record at its partition's next position: every partition's records end up contiguous. */
	void part_prologue() {
		const PartPlan& pp = st.part;
		const int NP = pp.P;
		o << part_ctl_decl();
		o << "  uint32_t* const pcnt = " << Pptr(pp.cnt, "uint32_t*") << ";\n";
		if (part_hist) {
			smem_sink = (size_t)NP * 8;
			o << "  uint32_t* const shist = (uint32_t*)vd_smem;\n";
			o << "  for (int i = threadIdx.x; i < " << NP << "; i += blockDim.x) { shist[i] = 0u; }\n";
			o << "  vd::block_sync();\n";
			return;
		}
		const std::string RT = rec_type();
		smem_sink = pp.smem1;
		o << "  " << RT << "* const pbuf = " << Pptr(pp.buf, RT + "*") << ";\n";
		o << "  const uint32_t pcap = (uint32_t)" << Pu((unsigned long long)pp.cap) << ";\n";
		o << "  uint32_t* const scur = (uint32_t*)vd_smem;\n";
		emit_pdl_wait();
		o << "  for (int q = threadIdx.x; q < " << NP << "; q += blockDim.x) {\n";
		o << "    const uint32_t c = __ldcg(&pcnt[(uint64_t)blockIdx.x * " << NP << "u + q]);\n";
		o << "    scur[q] = c != 0u ? (uint32_t)(__ldcg(&pstart[q]) + atomicAdd(&pcur[q], (unsigned long long)c)) : 0u;\n";
		o << "  }\n";
		o << "  vd::block_sync();\n";
	}

	/* pass 0: count the row into its partition.  Pass 1: write the row's record (the packed
	 * key, then each summed value minus its lower bound) at its partition's next position. */
	void part_row(const std::vector<Bounds>& kb) {
		const PartPlan& pp = st.part;
		const Sink& s = p.sink;
		o << "#pragma unroll\n    for (int v = 0; v < " << V << "; v++) {\n";
		o << "      if (act[v]) {\n";
		o << "        const uint64_t pk = " << packed_key(s.keys, kb, s.key_shift, "v") << ";\n";
		if (part_hist) {
			o << "        atomicAdd(&shist[" << part_of("pk") << "], 1u);\n";
			o << "      }\n    }\n";
			return;
		}
		o << "        uint64_t rw[2] = {pk, 0ull};\n";
		for (int a = 0; a < A(); a++) {
			if (s.aggs[a].count) {
				continue;
			}
			const std::string lo = P((unsigned long long)(int64_t)s.aggs[a].arg->b.lo);
			o << "        rw[" << pp.rec_word[a] << "] |= ((uint64_t)(" << expr(s.aggs[a].arg, "v") << ") - (uint64_t)" << lo
			  << ") << " << pp.rec_off[a] << ";\n";
		}
		o << "        const uint32_t at = atomicAdd(&scur[" << part_of("pk") << "], 1u);\n";
		o << "        if (at < pcap) {\n";
		if (pp.rec_words == 2) {
			o << "          pbuf[at] = make_ulonglong2(rw[0], rw[1]);\n";
		} else {
			o << "          pbuf[at] = rw[0];\n";
		}
		o << "        } else { atomicOr(err, VD_ERR_TABLE_FULL); }\n";
		o << "      }\n    }\n";
	}

	/* end of pass 0: the CTA's counts into its row of the count matrix and the totals; the
	 * last CTA writes the partition starts (exclusive prefix sums of the totals) */
	void part_epilogue() {
		const int NP = st.part.P;
		if (!part_hist) {
			return;
		}
		o << "  vd::block_sync();\n";
		o << "  for (int q = threadIdx.x; q < " << NP << "; q += blockDim.x) {\n";
		o << "    const uint32_t c = shist[q];\n";
		o << "    pcnt[(uint64_t)blockIdx.x * " << NP << "u + q] = c;\n";
		o << "    if (c != 0u) { atomicAdd(&ptot[q], (unsigned long long)c); }\n";
		o << "  }\n";
		o << "  __shared__ int hist_last;\n";
		o << "  __shared__ uint32_t hscan[33];\n";
		o << "  if (vd::last_block_done(&pctl[2], (unsigned long long)gridDim.x, &hist_last)) {\n";
		o << "    uint32_t* const stot = shist + " << NP << ";\n";
		o << "    for (int q = threadIdx.x; q < " << NP << "; q += blockDim.x) { stot[q] = (uint32_t)__ldcg(&ptot[q]); }\n";
		o << "    vd::block_sync();\n";
		o << "    vd::block_excl_scan(stot, shist, " << NP << ", hscan);\n";
		o << "    for (int q = threadIdx.x; q < " << NP << "; q += blockDim.x) { pstart[q] = shist[q]; }\n";
		o << "  }\n";
	}

	/* pass 2: the persistent aggregation kernel over work items (a partition's contiguous
	 * records, or an equal share of them for a partition holding more than R records) */
	std::string gen_part_aggregate() {
		const PartPlan& pp = st.part;
		const Sink& s = p.sink;
		const int NP = pp.P, S = pp.S, W = s.nwords, AT = pp.agg_threads;
		const int U = 4; /* record loads in flight per thread */
		const std::string RT = rec_type();
		std::ostringstream k;
		k << "extern \"C\" __global__ void __launch_bounds__(" << AT << ") " << name << "_extract(const VcParams p) {\n";
		k << "  vd::pdl_launch_dependents();\n  vd::pdl_wait();\n";
		k << "  unsigned* const err = (unsigned*)p.v[" << p.err_slot << "];\n";
		k << "  int64_t* const out = " << Pptr(qs.out, "int64_t*") << ";\n";
		k << "  const int64_t ocap = " << P((unsigned long long)qs.out_cap) << ";\n";
		k << "  unsigned long long* const ocount = " << Pptr(qs.out_count, "unsigned long long*") << ";\n";
		k << part_ctl_decl();
		k << "  const " << RT << "* __restrict__ pbuf = " << Pptr(pp.buf, "const " + RT + "*") << ";\n";
		k << "  uint32_t* const xkeys = " << Pptr(pp.skeys, "uint32_t*") << ";\n";
		k << "  unsigned long long* const xacc = " << Pptr(pp.sacc, "unsigned long long*") << ";\n";
		k << "  unsigned long long* const xitems = " << Pptr(pp.items, "unsigned long long*") << ";\n";
		k << "  const unsigned long long R = " << Pu((unsigned long long)pp.R) << ";\n";
		k << "  const unsigned long long xcap = " << Pu((unsigned long long)pp.scratch) << ";\n";
		k << "  extern __shared__ __align__(128) unsigned char vd_smem[];\n";
		k << "  uint32_t* const skeys = (uint32_t*)vd_smem;\n";
		k << "  unsigned long long* const sacc = (unsigned long long*)(vd_smem + " << (size_t)S * 4 << ");\n";
		k << "  uint32_t* const sk = (uint32_t*)(sacc + " << (size_t)S * W << ");\n";
		k << "  uint32_t* const sa = sk + " << NP << ";\n";
		k << "  uint32_t* const sb = sa + " << NP << ";\n";
		k << "  uint32_t* const ka = sb + " << NP << ";\n";
		k << "  uint32_t* const kb1 = ka + " << NP << ";\n";
		k << "  __shared__ uint32_t xscan[33];\n";
		k << "  __shared__ unsigned long long xres[1];\n";
		k << "  __shared__ uint32_t xitem, xlast;\n";
		k << "  __shared__ unsigned long long xrun;\n";
		k << "  for (int i = threadIdx.x; i < " << S << "; i += blockDim.x) { skeys[i] = 0u; }\n";
		k << "  for (int i = threadIdx.x; i < " << S * W << "; i += blockDim.x) { sacc[i] = 0ull; }\n";
		/* items: every split partition's items first (by partition), then the partitions that
		 * fit one item */
		k << "  for (int q = threadIdx.x; q < " << NP << "; q += blockDim.x) {\n";
		k << "    const unsigned long long t = __ldcg(&ptot[q]);\n";
		k << "    const uint32_t kq = (uint32_t)((t + R - 1ull) / R);\n";
		k << "    sk[q] = kq;\n    ka[q] = kq >= 2u ? kq : 0u;\n    kb1[q] = kq == 1u ? 1u : 0u;\n";
		k << "  }\n";
		k << "  vd::block_sync();\n";
		k << "  const uint32_t nA = vd::block_excl_scan(ka, sa, " << NP << ", xscan);\n";
		k << "  const uint32_t nB = vd::block_excl_scan(kb1, sb, " << NP << ", xscan);\n";
		k << "  for (;;) {\n";
		k << "    if (threadIdx.x == 0) { xitem = (uint32_t)atomicAdd(&pctl[0], 1ull); }\n";
		k << "    vd::block_sync();\n";
		k << "    const uint32_t item = xitem;\n";
		k << "    if (item >= nA + nB) { break; }\n";
		k << "    int q;\n    uint32_t j, kq;\n";
		k << "    if (item < nA) { q = vd::last_at_most(sa, " << NP << ", item); j = item - sa[q]; kq = sk[q]; }\n";
		k << "    else { q = vd::last_at_most(sb, " << NP << ", item - nA); j = 0u; kq = 1u; }\n";
		k << "    const unsigned long long t0 = __ldcg(&pstart[q]), tq = __ldcg(&ptot[q]);\n";
		k << "    const unsigned long long ra = t0 + tq * j / kq, rb = t0 + tq * (j + 1u) / kq;\n";
		k << "    for (unsigned long long base = ra; base < rb; base += (unsigned long long)blockDim.x * " << U << "u) {\n";
		k << "      " << RT << " r[" << U << "];\n      bool live[" << U << "];\n";
		k << "#pragma unroll\n      for (int u = 0; u < " << U << "; u++) {\n";
		k << "        const unsigned long long i = base + (unsigned long long)(u * blockDim.x + threadIdx.x);\n";
		k << "        live[u] = i < rb;\n";
		k << "        if (live[u]) { r[u] = __ldcs(&pbuf[i]); }\n";
		k << "      }\n";
		const std::string w0 = pp.rec_words == 2 ? "r[u].x" : "r[u]";
		const std::string w1 = pp.rec_words == 2 ? "r[u].y" : "r[u]";
		const unsigned long long kmask = (1ull << s.key_bits) - 1ull;
		k << "#pragma unroll\n      for (int u = 0; u < " << U << "; u++) {\n";
		k << "        const uint32_t pk = live[u] ? (uint32_t)(" << w0 << " & " << kmask << "ull) : 0xffffffffu;\n";
		{
			std::vector<PresumField> f;
			for (int a = 0; a < A(); a++) {
				if (s.aggs[a].count) {
					f.push_back({"", s.agg_word[a], s.agg_shift[a], 0, true});
					continue;
				}
				const int bits = span_bits(s.aggs[a].arg->b);
				const unsigned long long fmask = (1ull << bits) - 1ull;
				f.push_back({"(" + (pp.rec_word[a] == 1 ? w1 : w0) + " >> " + std::to_string(pp.rec_off[a]) + ") & " +
					std::to_string(fmask) + "ull", s.agg_word[a], s.agg_shift[a], bits, false});
			}
			emit_presum(k, "        ", "pk", "live[u]", f, W);
		}
		k << "        if (lead) {\n";
		k << "          const int sl = vd::st_find_or_insert(skeys, " << S << ", (uint32_t)vd::mix_hash32(pk), pk + 1u);\n";
		k << "          if (sl >= 0) {\n";
		k << "#pragma unroll\n            for (int a = 0; a < " << W << "; a++) { if (w[a]) { atomicAdd(&sacc[sl * " << W
		  << " + a], (unsigned long long)w[a]); } }\n";
		k << "          } else { atomicOr(err, VD_ERR_TABLE_FULL); }\n";
		k << "        }\n";
		k << "      }\n";
		k << "    }\n";
		k << "    vd::block_sync();\n";
		/* a split partition's item: leave the groups in a scratch run; the last item merges */
		k << "    bool emit = kq == 1u;\n";
		k << "    if (kq > 1u) {\n";
		k << "      uint32_t mine = 0u, ng;\n";
		k << "      for (int sl = threadIdx.x; sl < " << S << "; sl += blockDim.x) { mine += skeys[sl] != 0u ? 1u : 0u; }\n";
		k << "      const uint32_t pre = vd::block_excl_sum(mine, xscan, &ng);\n";
		k << "      if (threadIdx.x == 0) {\n";
		k << "        const unsigned long long x0 = atomicAdd(&pctl[1], (unsigned long long)ng);\n";
		k << "        if (x0 + ng > xcap) { atomicOr(err, VD_ERR_TABLE_FULL); ng = 0u; }\n";
		k << "        xrun = (x0 << 16) | ng;\n";
		k << "        xitems[item] = xrun;\n";
		k << "      }\n";
		k << "      vd::block_sync();\n";
		k << "      const unsigned long long x0 = xrun >> 16;\n";
		k << "      const uint32_t nrun = (uint32_t)(xrun & 0xffffull);\n";
		k << "      uint32_t wpos = pre;\n";
		k << "      for (int sl = threadIdx.x; sl < " << S << "; sl += blockDim.x) {\n";
		k << "        const uint32_t key = skeys[sl];\n";
		k << "        if (key == 0u) { continue; }\n";
		k << "        if (wpos < nrun) {\n";
		k << "          xkeys[x0 + wpos] = key;\n";
		k << "#pragma unroll\n          for (int a = 0; a < " << W << "; a++) { xacc[(x0 + wpos) * " << W << "ull + a] = sacc[sl * "
		  << W << " + a]; }\n";
		k << "        }\n";
		k << "        wpos++;\n";
		k << "      }\n";
		k << "      __threadfence();\n";
		k << "      vd::block_sync();\n";
		k << "      if (threadIdx.x == 0) { xlast = atomicAdd(&pdone[q], 1u) == kq - 1u ? 1u : 0u; }\n";
		k << "      vd::block_sync();\n";
		k << "      if (xlast) {\n";
		k << "        __threadfence();\n";
		k << "        for (uint32_t it = sa[q]; it < sa[q] + kq; it++) {\n";
		k << "          if (it == item) { continue; }\n";
		k << "          const unsigned long long run = __ldcg(&xitems[it]);\n";
		k << "          const unsigned long long b2 = run >> 16;\n";
		k << "          const uint32_t n2 = (uint32_t)(run & 0xffffull);\n";
		k << "          for (uint32_t e = threadIdx.x; e < n2; e += blockDim.x) {\n";
		k << "            const uint32_t key = __ldcg(&xkeys[b2 + e]);\n";
		k << "            const int sl = vd::st_find_or_insert(skeys, " << S << ", (uint32_t)vd::mix_hash32(key - 1u), key);\n";
		k << "            if (sl >= 0) {\n";
		k << "#pragma unroll\n              for (int a = 0; a < " << W << "; a++) {\n";
		k << "                const unsigned long long wv = __ldcg(&xacc[(b2 + e) * " << W << "ull + a]);\n";
		k << "                if (wv) { atomicAdd(&sacc[sl * " << W << " + a], wv); }\n";
		k << "              }\n";
		k << "            } else { atomicOr(err, VD_ERR_TABLE_FULL); }\n";
		k << "          }\n";
		k << "        }\n";
		k << "        vd::block_sync();\n";
		k << "        emit = true;\n";
		k << "      } else {\n";
		k << "        for (int i = threadIdx.x; i < " << S << "; i += blockDim.x) {\n";
		k << "          if (skeys[i] != 0u) {\n            skeys[i] = 0u;\n";
		k << "#pragma unroll\n            for (int a = 0; a < " << W << "; a++) { sacc[i * " << W << " + a] = 0ull; }\n";
		k << "          }\n        }\n";
		k << "        vd::block_sync();\n";
		k << "      }\n";
		k << "    }\n";
		/* the partition's result rows, reserved with one atomic; the table is left clear */
		auto field = [&](int a) {
			const int bits = s.agg_bits[a];
			const unsigned long long mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1ull);
			return "((w[" + std::to_string(s.agg_word[a]) + "] >> " + std::to_string(s.agg_shift[a]) + ") & " +
				std::to_string(mask) + "ull)";
		};
		k << "    if (emit) {\n";
		k << "      uint32_t mine = 0u, ng;\n";
		k << "      for (int sl = threadIdx.x; sl < " << S << "; sl += blockDim.x) { mine += skeys[sl] != 0u ? 1u : 0u; }\n";
		k << "      const uint32_t pre = vd::block_excl_sum(mine, xscan, &ng);\n";
		k << "      if (threadIdx.x == 0) { xres[0] = ng ? atomicAdd(ocount, (unsigned long long)ng) : 0ull; }\n";
		k << "      vd::block_sync();\n";
		k << "      int64_t pos = (int64_t)xres[0] + (int64_t)pre;\n";
		k << "      for (int sl = threadIdx.x; sl < " << S << "; sl += blockDim.x) {\n";
		k << "        const uint32_t key = skeys[sl];\n";
		k << "        if (key == 0u) { continue; }\n";
		k << "        uint64_t w[" << W << "];\n";
		k << "#pragma unroll\n        for (int a = 0; a < " << W << "; a++) { w[a] = sacc[sl * " << W << " + a]; }\n";
		k << "        const bool take = (int64_t)" << field(s.count_idx) << " > 0;\n";
		k << "        if (take && pos < ocap) {\n";
		k << "          const int64_t cnt = (int64_t)" << field(s.count_idx) << ";\n";
		int col = 0;
		for (size_t kk = 0; kk < s.keys.size(); kk++, col++) {
			const std::string lo = P((unsigned long long)(int64_t)s.keys[kk]->b.lo);
			const int bits = (kk + 1 < s.keys.size() ? s.key_shift[kk + 1] : s.key_bits) - s.key_shift[kk];
			const unsigned long long mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1ull);
			k << "          out[" << col << " * ocap + pos] = " << lo << " + (int64_t)((((uint64_t)key - 1ull) >> "
			  << s.key_shift[kk] << ") & " << mask << "ull);\n";
		}
		for (int a = 0; a < A(); a++) {
			if (!s.aggs[a].visible) {
				continue;
			}
			if (s.aggs[a].count) {
				k << "          out[" << col << " * ocap + pos] = cnt;\n";
			} else {
				const std::string lo = P((unsigned long long)(int64_t)s.aggs[a].arg->b.lo);
				k << "          out[" << col << " * ocap + pos] = (int64_t)(" << field(a) << " + (uint64_t)" << lo
				  << " * (uint64_t)cnt);\n";
			}
			col++;
		}
		k << "        }\n";
		k << "        pos++;\n";
		k << "        skeys[sl] = 0u;\n";
		k << "#pragma unroll\n        for (int a = 0; a < " << W << "; a++) { sacc[sl * " << W << " + a] = 0ull; }\n";
		k << "      }\n";
		k << "      vd::block_sync();\n";
		k << "    }\n";
		k << "  }\n";
		k << "}\n\n";
		return k.str();
	}

	void sink_epilogue() {
		Sink& s = p.sink;
		switch (s.kind) {
		case Sink::AggGlobal:
			o << "  __shared__ int64_t red[32 * " << A() << "];\n";
			o << "  vd::block_sum<" << A() << ">(acc, red);\n";
			o << "  unsigned long long* const g = " << Pptr(st.sink_dev, "unsigned long long*") << ";\n";
			o << "  if (threadIdx.x == 0) {\n";
			o << "#pragma unroll\n    for (int a = 0; a < " << A() << "; a++) { if (acc[a]) atomicAdd(&g[a], (unsigned long long)acc[a]); }\n";
			o << "  }\n";
			publish_slots("g", 1);
			break;
		case Sink::AggDense:
			o << "  unsigned long long* const g = " << Pptr(st.sink_dev, "unsigned long long*") << ";\n";
			if (private_acc) {
				/* fold the private accumulators into the block's slot array: one warp per
				 * (code, aggregate) pair, lanes striding over the threads' copies */
				o << "  vd::block_sync();\n";
				o << "  {\n    const int ng = min(*pncodes, " << kGmax << ");\n";
				o << "    for (int pr = (int)(threadIdx.x >> 5); pr < ng * " << A() << "; pr += (int)(blockDim.x >> 5)) {\n";
				o << "      int64_t sum = 0;\n";
				o << "      for (int t2 = (int)(threadIdx.x & 31); t2 < " << T << "; t2 += 32) { sum += priv[pr * " << T
				  << " + t2]; }\n";
				o << "#pragma unroll\n      for (int o2 = 16; o2 > 0; o2 >>= 1) { sum += (int64_t)__shfl_xor_sync(0xffffffffu, "
				     "(unsigned long long)sum, o2); }\n";
				o << "      if ((threadIdx.x & 31) == 0 && sum) { atomicAdd(&sacc[(int64_t)pcodes[pr / " << A() << "] * " << A()
				  << " + pr % " << A() << "], (unsigned long long)sum); }\n";
				o << "    }\n  }\n";
			}
			if (dense_in_smem) {
				const int64_t D = (int64_t)s.domain;
				o << "  vd::block_sync();\n";
				o << "  for (int64_t i = threadIdx.x; i < " << P((unsigned long long)D) << "; i += blockDim.x) {\n";
				o << "    unsigned long long sum[" << A() << "];\n";
				o << "#pragma unroll\n    for (int a = 0; a < " << A() << "; a++) { sum[a] = 0ull; }\n";
				o << "    for (int r = 0; r < " << replicas << "; r++) {\n";
				o << "#pragma unroll\n      for (int a = 0; a < " << A() << "; a++) { sum[a] += sacc0[(r * "
				  << P((unsigned long long)D) << " + i) * " << A() << " + a]; }\n";
				o << "    }\n";
				o << "    if (sum[" << s.count_idx << "]) {\n";
				o << "#pragma unroll\n      for (int a = 0; a < " << A() << "; a++) { atomicAdd(&g[i * " << A()
				  << " + a], sum[a]); }\n";
				o << "    }\n  }\n";
			}
			publish_slots("g", (int64_t)s.domain);
			break;
		case Sink::AggHash:
			if (part()) {
				part_epilogue();
				break;
			}
			if (gcache()) {
				const std::string K = gkey_type();
				const int W = s.nwords;
				o << "  vd::block_sync();\n";
				o << "  for (int i = threadIdx.x; i < " << cache_slots << "; i += blockDim.x) {\n";
				o << "    const " << K << " sk = ckeys[i];\n";
				o << "    if (sk != 0) {\n";
				o << "      uint64_t w[" << W << "];\n";
				o << "#pragma unroll\n      for (int a = 0; a < " << W << "; a++) { w[a] = cacc[i * " << W << " + a]; }\n";
				o << "      const uint64_t pk = (uint64_t)sk - 1ull;\n";
				if (gdirect()) {
					o << "      vd::gt_add<" << W << ">(gacc, (int64_t)pk, w);\n";
					o << "    }\n  }\n";
					break;
				}
				std::string h;
				for (size_t k = 0; k < s.keys.size(); k++) {
					const int bits = (k + 1 < s.keys.size() ? s.key_shift[k + 1] : s.key_bits) - s.key_shift[k];
					const unsigned long long mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1ull);
					const std::string kv = "(" + P((unsigned long long)(int64_t)s.keys[k]->b.lo) + " + (int64_t)((pk >> " +
						P((unsigned long long)s.key_shift[k]) + ") & " + Pu(mask) + "))";
					h = k == 0 ? "vd::hash(" + kv + ")" : "vd::rehash(" + h + ", " + kv + ")";
				}
				if (fl.hash != "voila") {
					h = s.key_bits <= 32 ? "vd::mix_hash32((uint32_t)pk)" : "vd::mix_hash64(pk)";
				}
				o << "      const int64_t slot = vd::gt_find_or_insert<" << K << ">(gkeys, gbmask, " << h << ", sk, err);\n";
				o << "      if (slot >= 0) { vd::gt_add<" << W << ">(gacc, slot, w); }\n";
				o << "    }\n  }\n";
			}
			break;
		default:
			break;
		}
	}

	/* ------------------------------------------------------------ extra kernels ---- */

	/* staged join build: clear the table for the materialised count, then insert */
	std::string gen_join_build() {
		JoinDesc& jd = plan.joins[p.sink.join];
		const std::string KT = jd.key64 ? "uint64_t" : "uint32_t";
		const std::string PT = jd.pay64 ? "uint64_t" : "uint32_t";
		const std::string S = join_slot_type(jd);
		std::ostringstream k;
		const std::string words = Pptr(jd.words, "unsigned long long*");
		const std::string table = Pptr(jd.table, S + "*");
		k << "extern \"C\" __global__ void __launch_bounds__(256) " << name << "_clear(const VcParams p) {\n";
		k << "  vd::pdl_launch_dependents();\n  vd::pdl_wait();\n";
		k << "  unsigned long long* const words = " << words << ";\n";
		k << "  " << S << "* const jt = " << table << ";\n";
		k << "  const uint64_t nb = vd::join_buckets<" << S << ">(words[0]);\n";
		k << "  if (blockIdx.x == 0 && threadIdx.x == 0) { words[1] = nb - 1; }\n";
		k << "  const uint64_t nslots = nb * vd::slots_per_bucket<" << S << ">();\n";
		k << "  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nslots; i += (uint64_t)gridDim.x * blockDim.x) {\n";
		k << "    jt[i].key = 0; jt[i].pay = 0;\n  }\n}\n\n";
		k << "extern \"C\" __global__ void __launch_bounds__(256) " << name << "_insert(const VcParams p) {\n";
		k << "  vd::pdl_launch_dependents();\n  vd::pdl_wait();\n";
		k << "  unsigned long long* const words = " << words << ";\n";
		k << "  " << S << "* const jt = " << table << ";\n";
		k << "  const " << KT << "* const skeys = " << Pptr(jd.stage_keys, "const " + KT + "*") << ";\n";
		k << "  const " << PT << "* const spay = " << Pptr(jd.stage_pay, "const " + PT + "*") << ";\n";
		k << "  const uint64_t* const shash = " << Pptr(st.stage_hash, "const uint64_t*") << ";\n";
		k << "  unsigned* const err = (unsigned*)p.v[" << p.err_slot << "];\n";
		k << "  const uint64_t cnt = words[0];\n";
		k << "  const uint64_t bmask = vd::join_buckets<" << S << ">(cnt) - 1;\n";
		k << "  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (uint64_t)gridDim.x * blockDim.x) {\n";
		k << "    vd::join_insert(jt, bmask, shash[i], skeys[i], spay[i], err" << (jd.join01 ? "" : ", bmask + 1ull")
		  << ");\n  }\n}\n\n";
		return k.str();
	}

	/* Hash-group extraction: rows with count > 0, keys unpacked, each visible aggregate's field
	 * taken out of its word and un-biased (sum = field + lo * count).  Every slot it reads is
	 * zeroed again, so the table is clear for the next run without a memset. */
	std::string gen_extract() {
		Sink& s = p.sink;
		std::ostringstream k;
		if (item) {
			k << "__device__ __noinline__ void " << name
			  << "_extract(const unsigned long long* __restrict__ pv, int64_t t_begin, int64_t t_end, int64_t nitems) {\n";
			k << "  const struct { const unsigned long long* __restrict__ v; } p = {pv};\n";
			k << "  (void)nitems;\n";
		} else {
			k << "extern \"C\" __global__ void __launch_bounds__(256) " << name << "_extract(const VcParams p) {\n";
			k << "  vd::pdl_launch_dependents();\n  vd::pdl_wait();\n";
		}
		const std::string K = gkey_type();
		const int W = s.nwords;
		k << "  int64_t* const out = " << Pptr(qs.out, "int64_t*") << ";\n";
		k << "  const int64_t ocap = " << P((unsigned long long)qs.out_cap) << ";\n";
		k << "  unsigned long long* const ocount = " << Pptr(qs.out_count, "unsigned long long*") << ";\n";
		if (!gdirect()) {
			k << "  " << K << "* const gkeys = " << Pptr(st.sink_dev, K + "*") << ";\n";
		}
		k << "  unsigned long long* const gacc = " << Pptr(st.sink_acc, "unsigned long long*") << ";\n";
		k << "  const int64_t nslots = " << P((unsigned long long)st.sink_cap) << ";\n";
		/* a block takes chunks of blockDim.x * kExtractK slots (slot q * blockDim.x + thread of
		 * the chunk); all keys of a chunk are loaded (from L2, coherent) before any is used */
		k << "  const int64_t chunk = (int64_t)blockDim.x * " << kExtractK << ";\n";
		if (item) {
			/* one item = chunks [t_begin, t_end) */
			k << "  const int64_t clim = (nslots + chunk - 1) / chunk;\n";
			k << "  for (int64_t ch = t_begin; ch < (t_end < clim ? t_end : clim); ch++) {\n";
		} else {
			k << "  for (int64_t ch = blockIdx.x; ch * chunk < nslots; ch += gridDim.x) {\n";
		}
		k << "    const int64_t cb = ch * chunk;\n";
		k << "    " << K << " kw[" << kExtractK << "];\n";
		k << "#pragma unroll\n    for (int q = 0; q < " << kExtractK << "; q++) {\n";
		k << "      const int64_t i = cb + (int64_t)q * blockDim.x + threadIdx.x;\n";
		if (gdirect()) {
			/* a direct table's slot is its packed key */
			k << "      kw[q] = i < nslots ? (" << K << ")(i + 1) : (" << K << ")0;\n";
		} else {
			k << "      kw[q] = i < nslots ? __ldcg(&gkeys[i]) : (" << K << ")0;\n";
		}
		k << "    }\n";
		k << "    uint64_t w[" << kExtractK << "][" << W << "];\n";
		k << "    bool take[" << kExtractK << "];\n";
		auto field = [&](int a) {
			const int bits = s.agg_bits[a];
			const unsigned long long mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1ull);
			return "((w[q][" + std::to_string(s.agg_word[a]) + "] >> " + std::to_string(s.agg_shift[a]) + ") & " +
				std::to_string(mask) + "ull)";
		};
		/* every word of the chunk is loaded before any slot is cleared (the clears would
		 * otherwise order each load after the previous slot's stores) */
		k << "#pragma unroll\n    for (int q = 0; q < " << kExtractK << "; q++) {\n";
		k << "      const int64_t i = cb + (int64_t)q * blockDim.x + threadIdx.x;\n";
		k << "#pragma unroll\n      for (int a = 0; a < " << W << "; a++) { w[q][a] = kw[q] != 0 ? __ldcg(&gacc[i * " << W
		  << " + a]) : 0ull; }\n";
		k << "    }\n";
		/* each warp reserves its rows with one atomic; for every q the lanes' rows are
		 * consecutive (ballot order), so the result columns are written coalesced */
		k << "    unsigned bal[" << kExtractK << "];\n    int wtot = 0;\n";
		k << "#pragma unroll\n    for (int q = 0; q < " << kExtractK << "; q++) {\n";
		k << "      const int64_t i = cb + (int64_t)q * blockDim.x + threadIdx.x;\n";
		k << "      take[q] = kw[q] != 0 && (int64_t)" << field(s.count_idx) << " > 0;\n";
		k << "      bal[q] = __ballot_sync(0xffffffffu, take[q]);\n";
		k << "      wtot += __popc(bal[q]);\n";
		if (gdirect()) {
			/* a used slot has a non-zero count */
			k << "      if (take[q]) {\n";
		} else {
			k << "      if (kw[q] != 0) {\n        gkeys[i] = 0;\n";
		}
		k << "#pragma unroll\n        for (int a = 0; a < " << W << "; a++) { gacc[i * " << W << " + a] = 0ull; }\n      }\n";
		k << "    }\n";
		k << "    unsigned long long wbase = 0ull;\n";
		k << "    if (vd::lane_id() == 0u && wtot > 0) { wbase = atomicAdd(ocount, (unsigned long long)wtot); }\n";
		k << "    wbase = __shfl_sync(0xffffffffu, wbase, 0);\n";
		k << "    int64_t woff = 0;\n";
		k << "#pragma unroll\n    for (int q = 0; q < " << kExtractK << "; q++) {\n";
		k << "    const int64_t pos = (int64_t)wbase + woff + __popc(bal[q] & vd::lanemask_lt());\n";
		k << "    woff += __popc(bal[q]);\n";
		k << "    if (take[q] && pos < ocap) {\n";
		k << "      const int64_t cnt = (int64_t)" << field(s.count_idx) << ";\n";
		int col = 0;
		for (size_t kk = 0; kk < s.keys.size(); kk++, col++) {
			const std::string lo = P((unsigned long long)(int64_t)s.keys[kk]->b.lo);
			const int bits = (kk + 1 < s.keys.size() ? s.key_shift[kk + 1] : s.key_bits) - s.key_shift[kk];
			const unsigned long long mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1ull);
			k << "      out[" << col << " * ocap + pos] = " << lo << " + (int64_t)((((uint64_t)kw[q] - 1ull) >> "
			  << P((unsigned long long)s.key_shift[kk]) << ") & " << Pu(mask) << ");\n";
		}
		for (int a = 0; a < A(); a++) {
			if (!s.aggs[a].visible) {
				continue;
			}
			if (s.aggs[a].count) {
				k << "      out[" << col << " * ocap + pos] = cnt;\n";
			} else {
				const std::string lo = P((unsigned long long)(int64_t)s.aggs[a].arg->b.lo);
				k << "      out[" << col << " * ocap + pos] = (int64_t)(" << field(a) << " + (uint64_t)" << lo
				  << " * (uint64_t)cnt);\n";
			}
			col++;
		}
		k << "    }\n    }\n  }\n}\n\n";
		return k.str();
	}
};

} // namespace

GeneratedCode generate_cuda(LoweredPlan& plan, const Flavor& fl, std::vector<PipeDeviceState>& st,
	const QueryDeviceState& qs, std::vector<std::vector<unsigned long long>>& params)
{
	GeneratedCode gc;
	std::ostringstream src;
	src << "#include \"voila_device.cuh\"\n";
	params.assign(plan.pipes.size(), {});
	for (auto& p : plan.pipes) {
		auto& prm = params[p.id];
		/* a pipeline feeding a later one writes its rows to its intermediate table */
		QueryDeviceState target = qs;
		if (p.out_inter >= 0) {
			const InterTable& it = plan.inters[p.out_inter];
			target.out = it.out;
			target.out_cap = it.cap;
			target.out_count = it.count;
		}
		const Flavor pfl = fl.for_pipe(p.id);
		PipeGen g(p, plan, pfl, st[p.id], target, prm);
		std::string main = g.gen_main();
		const size_t main_smem = g.smem_total;
		std::string hist;
		size_t hist_smem = 0;
		if (g.part()) {
			/* the partitioned group-by's histogram pass: the same pipeline, counting rows per
			 * partition */
			g.o.str("");
			g.o.clear();
			g.smem_total = 0;
			g.smem_sink = 0;
			g.part_hist = true;
			hist = g.gen_main();
			hist_smem = g.smem_total;
			g.part_hist = false;
			g.smem_total = main_smem;
		}
		std::string extra;
		if (p.sink.kind == Sink::JoinBuild && !plan.joins[p.sink.join].direct) {
			extra = g.gen_join_build();
		} else if (p.sink.kind == Sink::AggHash) {
			extra = g.part() ? g.gen_part_aggregate() : g.gen_extract();
		}
		src << "#define VcParams VcParams" << p.id << "\n";
		src << "struct VcParams" << p.id << " { unsigned long long v[" << std::max<size_t>(prm.size(), 1) << "]; };\n";
		src << hist << main << extra;
		src << "#undef VcParams\n\n";

		int hist_launch = -1;
		if (!hist.empty()) {
			Launch h;
			h.kernel = g.name + "_hist";
			h.pipe = p.id;
			h.stage = 0;
			h.smem = hist_smem;
			h.threads = pfl.threads;
			const int64_t htile = (int64_t)pfl.threads * pfl.rows;
			h.grid_items = std::max<int64_t>((p.rows + htile - 1) / htile, 1);
			h.grid_cap = st[p.id].part.max_ctas;
			hist_launch = (int)gc.launches.size();
			gc.launches.push_back(h);
		}
		Launch m;
		m.kernel = g.name + "_main";
		m.pipe = p.id;
		m.stage = 0;
		m.smem = g.smem_total;
		m.threads = pfl.threads;
		const int64_t tile = (int64_t)pfl.threads * pfl.rows;
		m.grid_items = std::max<int64_t>((p.rows + tile - 1) / tile, 1);
		m.dominant = p.id == plan.result_pipe;
		if (hist_launch >= 0) {
			m.grid_with = hist_launch;
			m.grid_cap = st[p.id].part.max_ctas;
		}
		if (p.sink.kind == Sink::AggGlobal || p.sink.kind == Sink::AggDense) {
			/* the last-block publication needs every launched block to count itself */
			m.grid_items = std::max<int64_t>(m.grid_items, 1);
		}
		gc.launches.push_back(m);
		if (p.sink.kind == Sink::JoinBuild && !plan.joins[p.sink.join].direct) {
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
		} else if (p.sink.kind == Sink::AggHash) {
			Launch e;
			e.kernel = g.name + "_extract";
			e.pipe = p.id;
			e.stage = 1;
			if (g.part()) {
				/* persistent: work items are taken from a counter */
				e.threads = st[p.id].part.agg_threads;
				e.smem = st[p.id].part.smem2;
				e.grid_items = 0;
			} else {
				e.threads = 256;
				e.grid_items = (st[p.id].sink_cap + 256 * 4 - 1) / (256 * 4);
			}
			gc.launches.push_back(e);
		}
	}
	gc.source = src.str();
	return gc;
}

/*
 * Batch code: every pipeline of every query becomes a device item function (deduplicated by
 * generated text, so instances of one shape share code) and a list of work items over its
 * tiles.  Items are ordered by dependency level and carry the done-counter they must wait
 * for, so the persistent kernel's queue runs them in dependency order:
 *   level L of a query's join builds: a build pipeline that probes no join is level 0; one
 *     whose rows probe other joins (a build side that is itself a join chain) is one level
 *     above the builds of those joins.  Level-0 builds wait for the query's state clears
 *     (dep_target -2, patched by the runtime with their count), level-L builds for every
 *     item of level L-1;
 *   the query's other pipelines (probes, aggregations, emits) wait for the top build level;
 *   group extraction waits for its group-by pipeline.
 * The queue concatenates the phases in level order across queries, so an item only ever
 * waits for items earlier in the queue.  Counter 0 is the queue head, counter 1 counts
 * finished clears.
 */
BatchCode generate_batch(std::vector<Query*>& queries, const std::vector<Flavor>& flavors, int threads,
	int64_t tiles_per_item)
{
	BatchCode bc;
	std::map<std::string, int> shape_of;
	std::vector<std::string> shape_fn;
	std::ostringstream funcs;
	std::vector<std::vector<BatchItem>> phases;
	auto phase_list = [&](size_t ph) -> std::vector<BatchItem>& {
		if (ph >= phases.size()) {
			phases.resize(ph + 1);
		}
		return phases[ph];
	};
	int ncounters = 2;
	auto add_shape = [&](const std::string& text, const std::string& suffix) -> int {
		auto it = shape_of.find(text);
		if (it != shape_of.end()) {
			return it->second;
		}
		const int id = (int)shape_fn.size();
		const std::string fname = "vc_s" + std::to_string(id);
		std::string t = text;
		for (size_t pos = t.find("VCSHAPE"); pos != std::string::npos; pos = t.find("VCSHAPE", pos)) {
			t.replace(pos, 7, fname);
		}
		funcs << t;
		shape_fn.push_back(fname + suffix);
		shape_of[text] = id;
		return id;
	};
	for (size_t qi = 0; qi < queries.size(); qi++) {
		Query& q = *queries[qi];
		QueryState& st = state_of(q);
		bc.query_params_begin.push_back((int64_t)bc.params.size());
		/* every CTA of the persistent kernel reserves the largest shape's shared memory, so
		 * the knobs that need much of it run as their lean equivalents inside a batch */
		auto batch_flavor = [&](int pipe) {
			Flavor f = flavors[qi].for_pipe(pipe);
			f.threads = threads;
			f.load = "ldg";
			if (f.lowcard == "private" || f.lowcard == "regs" || f.lowcard == "packed") {
				f.lowcard = "combine";
			}
			f.cache_slots = std::min(f.cache_slots, 256);
			if (f.aggr == "part") {
				/* two passes with a data-dependent item count: the global group table instead */
				f.aggr = "global";
			}
			f.sink_smem = std::min(f.sink_smem, 16 * 1024);
			return f;
		};
		QueryDeviceState qs;
		qs.out = q.out;
		qs.out_cap = q.out_cap;
		qs.out_count = q.out_count;
		auto tile_of = [&](const Pipeline& p) {
			const Flavor f = batch_flavor(p.id);
			return (int64_t)f.threads * f.rows;
		};
		auto items_of = [&](const Pipeline& p) {
			const int64_t ntiles = std::max<int64_t>((p.rows + tile_of(p) - 1) / tile_of(p), 1);
			return (ntiles + tiles_per_item - 1) / tiles_per_item;
		};
		if (!q.plan.inters.empty()) {
			throw Error(6, "batched queries cannot hold aggregations below the plan root yet");
		}
		/* dependency levels of the join builds, and the work items per level */
		std::vector<int> level(q.plan.pipes.size(), 0);
		std::map<int, int> build_pipe_of_join;
		int top_level = -1;
		for (auto& p : q.plan.pipes) {
			if (p.sink.kind == Sink::JoinBuild && !q.plan.joins[p.sink.join].direct) {
				throw Error(6, "batched queries need direct join builds (build=staged is not batchable)");
			}
			int lv = 0;
			for (auto& op : p.ops) {
				if (op.kind == Op::Probe) {
					auto b = build_pipe_of_join.find(op.join);
					if (b == build_pipe_of_join.end()) {
						throw Error(6, "batch: a pipeline probes a join whose build pipeline comes later");
					}
					lv = std::max(lv, level[b->second] + 1);
				}
			}
			level[p.id] = lv;
			if (p.sink.kind == Sink::JoinBuild) {
				build_pipe_of_join[p.sink.join] = p.id;
				top_level = std::max(top_level, lv);
			}
		}
		std::vector<int> level_counter(top_level + 1, -1);
		std::vector<int64_t> level_items(top_level + 1, 0);
		for (auto& p : q.plan.pipes) {
			if (p.sink.kind == Sink::JoinBuild) {
				if (level_counter[level[p.id]] < 0) {
					level_counter[level[p.id]] = ncounters++;
				}
				level_items[level[p.id]] += items_of(p);
			}
		}
		for (auto& p : q.plan.pipes) {
			std::vector<unsigned long long> prm;
			/* the query keeps its own parameter layout for standalone runs */
			const int saved_err = p.err_slot;
			const std::vector<int> saved_cols = p.col_slots;
			if (p.sink.kind == Sink::AggHash && !st.pipes[p.id].sink_dev) {
				throw Error(6, "batch: a partitioned group-by has no group table");
			}
			const Flavor pfl = batch_flavor(p.id);
			PipeGen g(p, q.plan, pfl, st.pipes[p.id], qs, prm);
			g.item = true;
			g.name = "VCSHAPE";
			const std::string main_src = g.gen_main();
			const std::string extract_src = p.sink.kind == Sink::AggHash ? g.gen_extract() : std::string();
			bc.smem = std::max(bc.smem, g.smem_total);
			prm[p.err_slot] = (unsigned long long)(uintptr_t)q.err;
			for (size_t c = 0; c < p.cols.size(); c++) {
				prm[p.col_slots[c]] = (unsigned long long)(uintptr_t)column_dev(q, p.cols[c]);
			}
			p.err_slot = saved_err;
			p.col_slots = saved_cols;
			const int64_t poff = (int64_t)bc.params.size();
			bc.params.insert(bc.params.end(), prm.begin(), prm.end());

			const int sid = add_shape(main_src, "_main");
			const int64_t ntiles = std::max<int64_t>((p.rows + tile_of(p) - 1) / tile_of(p), 1);
			const int64_t nit = items_of(p);
			const bool is_build = p.sink.kind == Sink::JoinBuild;
			/* phase (position in the queue), the counter waited for and its target */
			size_t phase;
			int dep, counter;
			int64_t dep_target;
			if (is_build) {
				const int lv = level[p.id];
				phase = (size_t)lv;
				counter = level_counter[lv];
				dep = lv == 0 ? 1 : level_counter[lv - 1];
				dep_target = lv == 0 ? -2 : level_items[lv - 1];
			} else {
				phase = (size_t)(top_level + 1);
				counter = ncounters++;
				dep = top_level < 0 ? 1 : level_counter[top_level];
				dep_target = top_level < 0 ? -2 : level_items[top_level];
			}
			for (int64_t k = 0; k < nit; k++) {
				BatchItem it;
				it.shape = sid;
				it.params = poff;
				it.begin = k; /* tiles k, k + nit, k + 2 nit, ... (the item functions stride by nitems) */
				it.end = ntiles;
				it.nitems = nit;
				it.dep = dep;
				it.dep_target = dep_target;
				it.done = counter;
				it.finish = (!is_build && p.sink.kind != Sink::AggHash) ? (int)qi : -1;
				phase_list(phase).push_back(it);
			}
			if (p.sink.kind == Sink::AggHash) {
				const int sid2 = add_shape(extract_src, "_extract");
				const int64_t group = (int64_t)threads * 4;
				const int64_t ngroups = std::max<int64_t>((st.pipes[p.id].sink_cap + group - 1) / group, 1);
				const int64_t per = std::max<int64_t>(tiles_per_item / 4, 1);
				const int64_t nit2 = (ngroups + per - 1) / per;
				const int counter2 = ncounters++;
				for (int64_t k = 0; k < nit2; k++) {
					BatchItem it;
					it.shape = sid2;
					it.params = poff;
					it.begin = k * per;
					it.end = std::min((k + 1) * per, ngroups);
					it.nitems = nit2;
					it.dep = counter;
					it.dep_target = nit;
					it.done = counter2;
					it.finish = (int)qi;
					phase_list(phase + 1).push_back(it);
				}
			}
		}
	}
	/* Within a phase, each pipeline's items stay together (its hash table stays in L2 while
	 * its items run; interleaving all pipelines' items thrashed L2 and slowed the group-bys
	 * by a third), largest pipelines first so the small ones fill the tail of the phase. */
	for (auto& ph : phases) {
		std::map<int64_t, std::vector<BatchItem>> by_stage; /* key: parameter offset and done counter */
		std::vector<int64_t> order;
		for (auto& it : ph) {
			const int64_t key = it.params * 4096 + it.done;
			if (!by_stage.count(key)) {
				order.push_back(key);
			}
			by_stage[key].push_back(it);
		}
		std::stable_sort(order.begin(), order.end(),
			[&](int64_t a, int64_t b) { return by_stage[a].size() > by_stage[b].size(); });
		for (int64_t k : order) {
			bc.items.insert(bc.items.end(), by_stage[k].begin(), by_stage[k].end());
		}
	}
	bc.query_params_begin.push_back((int64_t)bc.params.size());
	bc.ncounters = ncounters;

	std::ostringstream src;
	src << "#define VD_COHERENT_TABLES 1\n#include \"voila_device.cuh\"\n";
	src << "struct VcBatchItem { int shape; int dep; long long params; long long begin; long long end; "
		"long long nitems; long long dep_target; int done; int finish; };\n\n";
	src << funcs.str();
	/* the kernel holds every shape, so its register count is the largest shape's: bound it so
	 * that 32 warps per SM stay resident (the heaviest shapes spill a little instead) */
	const int min_blocks = std::max(1, 1024 / threads);
	src << "extern \"C\" __global__ void __launch_bounds__(" << threads << ", " << min_blocks
		<< ") vc_batch(const VcBatchItem* __restrict__ items, "
		"long long nwork, unsigned long long* counters, const unsigned long long* __restrict__ pool, "
		"unsigned long long* finish_ns, int nq, unsigned* err, unsigned long long wait_ns) {\n";
	src << "  __shared__ long long s_w;\n  __shared__ int s_ok;\n";
	src << "  if (threadIdx.x == 0) { atomicCAS(&finish_ns[nq], 0ull, (unsigned long long)vd::globaltimer_ns()); }\n";
	src << "  for (;;) {\n";
	src << "    if (threadIdx.x == 0) { s_w = (long long)atomicAdd(&counters[0], 1ull); }\n";
	src << "    vd::block_sync();\n";
	src << "    const long long w = s_w;\n";
	src << "    if (w >= nwork) { break; }\n";
	src << "    const VcBatchItem it = items[w];\n";
	src << "    if (threadIdx.x == 0) {\n";
	src << "      int ok = 1;\n";
	src << "      if (it.dep >= 0) {\n";
	src << "        uint64_t t0 = 0;\n";
	src << "        for (unsigned spin = 0; *(volatile unsigned long long*)&counters[it.dep] < (unsigned long long)it.dep_target; spin++) {\n";
	src << "          if (spin == 0) { t0 = vd::globaltimer_ns(); }\n";
	src << "          else if ((spin & 255u) == 0 && vd::globaltimer_ns() - t0 > wait_ns) { ok = 0; break; }\n";
	src << "          __nanosleep(100);\n";
	src << "        }\n";
	src << "        __threadfence();\n";
	src << "      }\n";
	src << "      s_ok = ok;\n";
	src << "    }\n";
	src << "    vd::block_sync();\n";
	src << "    if (s_ok) {\n";
	src << "      switch (it.shape) {\n";
	src << "      case -1: {\n";
	src << "        unsigned char* base = (unsigned char*)pool[it.params];\n";
	src << "        for (long long off = it.begin + (long long)threadIdx.x * 16; off < it.end; off += (long long)blockDim.x * 16) {\n";
	src << "          *(uint4*)(base + off) = make_uint4(0u, 0u, 0u, 0u);\n";
	src << "        }\n        break;\n      }\n";
	for (size_t s = 0; s < shape_fn.size(); s++) {
		src << "      case " << s << ": " << shape_fn[s] << "(pool + it.params, it.begin, it.end, it.nitems); break;\n";
	}
	src << "      default: break;\n      }\n";
	src << "    } else if (threadIdx.x == 0) {\n      atomicOr(err, VD_ERR_WAIT_TIMEOUT);\n    }\n";
	/* every thread's stores (payloads, results) are device-visible before the item counts
	 * as done */
	src << "    __threadfence();\n";
	src << "    vd::block_sync();\n";
	src << "    if (threadIdx.x == 0) {\n";
	src << "      __threadfence();\n";
	src << "      const unsigned long long old = atomicAdd(&counters[it.done], 1ull);\n";
	src << "      if (it.finish >= 0 && old + 1ull == (unsigned long long)it.nitems) { finish_ns[it.finish] = vd::globaltimer_ns(); }\n";
	src << "    }\n";
	src << "  }\n}\n";
	bc.source = src.str();
	return bc;
}

} // namespace vc
