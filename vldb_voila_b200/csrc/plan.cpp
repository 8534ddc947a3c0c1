/*
 * Plan text -> relational plan mirror -> lowered pipelines.
 *
 * The lowering follows the pipeline structure the reference's RelOpTranslator produces
 * (relalg_translator.cpp:169-1124), re-expressed for fused GPU pipelines:
 *   - Scan opens a pipeline over a base table (relalg_translator.cpp:202-272);
 *   - Select adds a filter (seltrue + emit, :343-378);
 *   - Project replaces the visible columns; later assignments may use earlier ones
 *     (:275-341, expr_cache);
 *   - HashJoin closes the build side's pipeline with a table-build sink (materialize +
 *     bucket_build, :828-931) and appends a probe to the probe side's pipeline; after it the
 *     visible columns are the probe side's, then the build keys (taking the probe key values,
 *     :965-975) and the build payloads (:1000-1012).  Join01 stops at the first match
 *     (:1032-1042);
 *   - HashAggr ends the pipeline with a group-by or global aggregation; a count is added
 *     when the plan has none (:469-472) and result rows are the groups whose count is > 0
 *     (:692-701).
 *
 * Typing: like the reference's typing pass (typing_pass.cpp:9-23, :164-176, :244-259) every
 * value carries an exact [lo, hi] range derived from the columns' declared min/max.  Here
 * all arithmetic runs in int64 and a plan whose ranges (or sums, bounded by the row count)
 * could leave int64 is rejected instead of being widened to 128 bits.
 */
#include <algorithm>
#include <climits>

#include "engine_internal.hpp"

namespace vc {

static const int kErrInvalid = 1;
static const int kErrUnsupported = 6;

/* ------------------------------------------------------------------ plan text ---------- */

static RelExprP parse_expr(const vc_sexpr::Node& n)
{
	auto e = std::make_shared<RelExpr>();
	const std::string& h = n.head();
	if (h == "const") {
		e->kind = RelExpr::Const;
		e->text = n.atom_text(1);
	} else if (h == "col") {
		e->kind = RelExpr::ColId;
		e->text = n.atom_text(1);
	} else if (h == "assign") {
		e->kind = RelExpr::Assign;
		e->text = n.atom_text(1);
		e->args.push_back(parse_expr(n.at(2)));
	} else if (h == "fun") {
		e->kind = RelExpr::Fun;
		e->text = n.atom_text(1);
		for (size_t i = 2; i < n.kids.size(); i++) {
			e->args.push_back(parse_expr(n.kids[i]));
		}
	} else {
		throw Error(kErrInvalid, "plan: unknown expression '" + h + "'");
	}
	return e;
}

static std::vector<RelExprP> parse_expr_list(const vc_sexpr::Node& n)
{
	if (n.atom) {
		throw Error(kErrInvalid, "plan: expected an expression list, got '" + n.text + "'");
	}
	std::vector<RelExprP> r;
	for (auto& k : n.kids) {
		r.push_back(parse_expr(k));
	}
	return r;
}

static RelOpP parse_op(const vc_sexpr::Node& n)
{
	auto op = std::make_shared<RelOp>();
	const std::string& h = n.head();
	if (h == "scan") {
		op->kind = RelOp::Scan;
		op->table = n.atom_text(1);
		const auto& cols = n.at(2);
		if (cols.atom) {
			throw Error(kErrInvalid, "plan: scan expects a column list");
		}
		for (auto& c : cols.kids) {
			if (!c.atom) {
				throw Error(kErrInvalid, "plan: scan columns must be names");
			}
			op->columns.push_back(c.text);
		}
	} else if (h == "select") {
		op->kind = RelOp::Select;
		op->predicate = parse_expr(n.at(1));
		op->left = parse_op(n.at(2));
	} else if (h == "project") {
		op->kind = RelOp::Project;
		op->exprs = parse_expr_list(n.at(1));
		op->left = parse_op(n.at(2));
	} else if (h == "aggr") {
		op->kind = RelOp::HashAggr;
		const std::string& v = n.atom_text(1);
		if (v != "hash" && v != "global") {
			throw Error(kErrInvalid, "plan: aggr variant must be hash or global");
		}
		op->global = v == "global";
		op->exprs = parse_expr_list(n.at(2));
		op->aggregates = parse_expr_list(n.at(3));
		op->left = parse_op(n.at(4));
	} else if (h == "join") {
		op->kind = RelOp::HashJoin;
		const std::string& v = n.atom_text(1);
		if (v != "join01" && v != "joinN") {
			throw Error(kErrInvalid, "plan: join variant must be join01 or joinN");
		}
		op->join01 = v == "join01";
		op->left_keys = parse_expr_list(n.at(2));
		op->left_payl = parse_expr_list(n.at(3));
		op->left = parse_op(n.at(4));
		op->right_keys = parse_expr_list(n.at(5));
		op->right_payl = parse_expr_list(n.at(6));
		op->right = parse_op(n.at(7));
		if (op->left_keys.empty() || op->left_keys.size() != op->right_keys.size()) {
			throw Error(kErrInvalid, "plan: join needs the same non-zero number of probe and build keys");
		}
	} else {
		throw Error(kErrInvalid, "plan: unknown operator '" + h + "'");
	}
	return op;
}

RelOpP parse_plan(const std::string& text)
{
	try {
		return parse_op(vc_sexpr::parse(text));
	} catch (const Error&) {
		throw;
	} catch (const std::exception& e) {
		throw Error(kErrInvalid, e.what());
	}
}

/* ------------------------------------------------------------------ bounds ------------- */

static const __int128 kI64Max = (__int128)INT64_MAX;
static const __int128 kI64Min = (__int128)INT64_MIN;

/* Gregorian year of a Julian day number: the conversion of the Calendar FAQ (C. Tondering),
 * in the unsigned 32-bit steps the reference uses (runtime.hpp:128-148) */
static int64_t julian_year(int64_t jd)
{
	const uint32_t a = (uint32_t)jd + 32044u;
	const uint32_t b = (4u * a + 3u) / 146097u;
	const uint32_t c = a - (146097u * b) / 4u;
	const uint32_t d = (4u * c + 3u) / 1461u;
	const uint32_t e = c - (1461u * d) / 4u;
	const uint32_t m = (5u * e + 2u) / 153u;
	return (int64_t)(100u * b + d - 4800u + m / 10u);
}

static void check_range(const Bounds& b, const std::string& what)
{
	if (b.lo < kI64Min || b.hi > kI64Max) {
		throw Error(kErrUnsupported, "value range of " + what + " exceeds int64; the CUDA flavor keeps "
			"every value and sum an exact int64");
	}
}

static int bits_for(__int128 range)
{
	/* bits needed to store values 0 .. range-1 */
	int b = 0;
	while (b < 127 && ((__int128)1 << b) < range) {
		b++;
	}
	return b;
}

/* ------------------------------------------------------------------ lowering ----------- */

namespace {

struct ScopeEntry {
	std::string name;
	BExprP e;
	std::string table, column; /* unresolved base column */
};

struct Scope {
	std::vector<ScopeEntry> cols;
	ScopeEntry* find(const std::string& n) {
		for (auto it = cols.rbegin(); it != cols.rend(); ++it) {
			if (it->name == n) {
				return &*it;
			}
		}
		return nullptr;
	}
};

struct Lowerer {
	std::map<std::string, Table>& tables;
	const Flavor& fl;
	const StringDict& dict;
	LoweredPlan out;

	std::map<std::string, Table> inter_tables; /* intermediate tables by name */
	int name_counter = 0; /* the reference translator's id counter (relalg_translator.hpp:26-30) */

	Lowerer(std::map<std::string, Table>& t, const Flavor& f, const StringDict& d) : tables(t), fl(f), dict(d) {}

	Table& table(const std::string& n) {
		auto ii = inter_tables.find(n);
		if (ii != inter_tables.end()) {
			return ii->second;
		}
		auto it = tables.find(n);
		if (it == tables.end()) {
			throw Error(kErrInvalid, "unknown table '" + n + "'");
		}
		return it->second;
	}

	BExprP resolve(ScopeEntry& s, Pipeline& p) {
		if (s.e) {
			return s.e;
		}
		Table& t = table(s.table);
		Column* c = t.find(s.column);
		if (!c) {
			throw Error(kErrInvalid, "unknown column '" + s.table + "." + s.column + "'");
		}
		auto e = std::make_shared<BExpr>();
		e->kind = BExpr::Col;
		e->col = -1;
		for (size_t i = 0; i < p.cols.size(); i++) {
			if (p.cols[i].table == s.table && p.cols[i].name == s.column) {
				e->col = (int)i;
			}
		}
		if (e->col < 0) {
			e->col = (int)p.cols.size();
			p.cols.push_back(PipeColumn{s.table, s.column, c->type, c->lo, c->hi, c->host});
		}
		e->b.lo = c->lo;
		e->b.hi = c->hi;
		e->str = c->str || c->type == VC_TYPE_STR;
		s.e = e;
		return e;
	}

	BExprP bind(const RelExprP& re, Scope& sc, Pipeline& p) {
		switch (re->kind) {
		case RelExpr::Const: {
			auto e = std::make_shared<BExpr>();
			e->kind = BExpr::Const;
			e->sval = re->text;
			try {
				size_t used = 0;
				e->cval = std::stoll(re->text, &used);
				if (used != re->text.size()) {
					throw std::invalid_argument("trailing");
				}
			} catch (const std::exception&) {
				/* not an integer: a string constant, usable against string columns */
				e->str = true;
				e->cval = 0;
			}
			e->b.lo = e->b.hi = e->cval;
			return e;
		}
		case RelExpr::ColId: {
			ScopeEntry* s = sc.find(re->text);
			if (!s) {
				throw Error(kErrInvalid, "cannot find '" + re->text + "' among the visible columns");
			}
			return resolve(*s, p);
		}
		case RelExpr::Assign:
			throw Error(kErrInvalid, "assign is only allowed in a projection list");
		case RelExpr::Fun:
			break;
		}
		if (re->text == "contains") {
			/* contains(string column, pattern) (runtime.hpp:150-224, kernel_generator.py:435-437):
			 * the set of dictionary codes whose strings hold the pattern, as a bitmap over the
			 * column's code range; the kernel tests the row's code */
			if (re->args.size() != 2) {
				throw Error(kErrInvalid, "contains takes two arguments");
			}
			BExprP col = bind(re->args[0], sc, p);
			BExprP pat = bind(re->args[1], sc, p);
			if (!col->str || col->kind == BExpr::Const || pat->kind != BExpr::Const) {
				throw Error(kErrUnsupported, "contains needs a string column and a constant pattern");
			}
			CodeBitmap bm;
			bm.lo = (int64_t)col->b.lo;
			const int64_t n = (int64_t)(col->b.hi - col->b.lo) + 1;
			bm.bits.assign((size_t)std::max<int64_t>((n + 31) / 32, 1), 0u);
			for (int64_t i = 0; i < n; i++) {
				const int64_t code = bm.lo + i;
				if (code >= 0 && code < (int64_t)dict.strings.size() &&
					dict.strings[(size_t)code].find(pat->sval) != std::string::npos) {
					bm.bits[(size_t)(i >> 5)] |= 1u << (i & 31);
				}
			}
			auto e = std::make_shared<BExpr>();
			e->kind = BExpr::Fun;
			e->fn = "inset";
			e->args.push_back(col);
			e->aux = (int)out.bitmaps.size();
			out.bitmaps.push_back(std::move(bm));
			e->boolean = true;
			e->b.lo = 0;
			e->b.hi = 1;
			return e;
		}
		if (re->text == "extract_year") {
			/* year of a date stored as its Julian day number (runtime.hpp:128-148); the
			 * bounds are the years of the date bounds (the conversion is monotonic) */
			if (re->args.size() != 1) {
				throw Error(kErrInvalid, "extract_year takes one argument");
			}
			auto e = std::make_shared<BExpr>();
			e->kind = BExpr::Fun;
			e->fn = "extract_year";
			e->args.push_back(bind(re->args[0], sc, p));
			const Bounds& a = e->args[0]->b;
			if (e->args[0]->boolean || a.lo < 0 || a.hi > 1000000000) {
				throw Error(kErrUnsupported, "extract_year needs a day number in [0, 1e9]");
			}
			e->b.lo = julian_year((int64_t)a.lo);
			e->b.hi = julian_year((int64_t)a.hi);
			return e;
		}
		static const std::map<std::string, std::string> names = {
			{"<=", "le"}, {"<", "lt"}, {">=", "ge"}, {">", "gt"}, {"=", "eq"}, {"!=", "ne"},
			{"+", "add"}, {"-", "sub"}, {"*", "mul"},
			{"le", "le"}, {"lt", "lt"}, {"ge", "ge"}, {"gt", "gt"}, {"eq", "eq"}, {"ne", "ne"},
			{"add", "add"}, {"sub", "sub"}, {"mul", "mul"}, {"and", "and"}, {"or", "or"}};
		auto it = names.find(re->text);
		if (it == names.end()) {
			throw Error(kErrUnsupported, "function '" + re->text + "' is not supported by the CUDA flavor");
		}
		auto e = std::make_shared<BExpr>();
		e->kind = BExpr::Fun;
		e->fn = it->second;
		for (auto& a : re->args) {
			e->args.push_back(bind(a, sc, p));
		}
		if (e->args.size() != 2) {
			throw Error(kErrInvalid, "function '" + re->text + "' takes two arguments");
		}
		if (e->args[0]->str || e->args[1]->str) {
			/* strings compare by dictionary code: only (in)equality, and a string constant is
			 * its code (-1, equal to no row, when the dictionary does not hold it) */
			if (e->fn != "eq" && e->fn != "ne") {
				throw Error(kErrUnsupported, "strings support =, != and contains only");
			}
			for (auto& x : e->args) {
				if (x->kind == BExpr::Const) {
					auto c = std::make_shared<BExpr>();
					c->kind = BExpr::Const;
					c->cval = dict.find(x->sval);
					c->b.lo = c->b.hi = c->cval;
					x = c;
				} else if (!x->str) {
					throw Error(kErrUnsupported, "a string compares only with a string");
				}
			}
		}
		const Bounds& a = e->args[0]->b;
		const Bounds& b = e->args[1]->b;
		if (e->fn == "add") {
			e->b.lo = a.lo + b.lo;
			e->b.hi = a.hi + b.hi;
		} else if (e->fn == "sub") {
			e->b.lo = a.lo - b.hi;
			e->b.hi = a.hi - b.lo;
		} else if (e->fn == "mul") {
			__int128 c[4] = {a.lo * b.lo, a.lo * b.hi, a.hi * b.lo, a.hi * b.hi};
			e->b.lo = *std::min_element(c, c + 4);
			e->b.hi = *std::max_element(c, c + 4);
		} else {
			e->boolean = true;
			e->b.lo = 0;
			e->b.hi = 1;
			if ((e->fn == "and" || e->fn == "or") && !(e->args[0]->boolean && e->args[1]->boolean)) {
				throw Error(kErrInvalid, "'" + re->text + "' needs two predicates");
			}
		}
		if (!e->boolean && (e->args[0]->boolean || e->args[1]->boolean)) {
			throw Error(kErrUnsupported, "arithmetic on predicates is not supported");
		}
		check_range(e->b, "'" + re->text + "'");
		return e;
	}

	/* Returns the index of the still-open pipeline that produces op's rows. */
	int lower(const RelOpP& op, Scope& sc) {
		switch (op->kind) {
		case RelOp::Scan: {
			Table& t = table(op->table);
			Pipeline p;
			p.id = (int)out.pipes.size();
			p.table = op->table;
			p.rows = t.rows;
			sc.cols.clear();
			for (auto& c : op->columns) {
				if (!t.find(c)) {
					throw Error(kErrInvalid, "unknown column '" + op->table + "." + c + "'");
				}
				sc.cols.push_back(ScopeEntry{op->table + "." + c, nullptr, op->table, c});
			}
			p.sink.kind = Sink::Emit;
			out.pipes.push_back(p);
			return p.id;
		}
		case RelOp::Select: {
			int pi = lower(op->left, sc);
			BExprP pred = bind(op->predicate, sc, out.pipes[pi]);
			if (!pred->boolean) {
				throw Error(kErrInvalid, "select predicate is not a comparison");
			}
			Op f;
			f.kind = Op::Filter;
			f.pred = pred;
			out.pipes[pi].ops.push_back(f);
			return pi;
		}
		case RelOp::Project: {
			int pi = lower(op->left, sc);
			Scope ns;
			Scope lookup = sc; /* earlier assignments become visible to later ones */
			for (auto& pe : op->exprs) {
				if (pe->kind == RelExpr::Assign) {
					BExprP e = bind(pe->args[0], lookup, out.pipes[pi]);
					ns.cols.push_back(ScopeEntry{pe->text, e, "", ""});
					lookup.cols.push_back(ScopeEntry{pe->text, e, "", ""});
				} else if (pe->kind == RelExpr::ColId) {
					ScopeEntry* s = lookup.find(pe->text);
					if (!s) {
						throw Error(kErrInvalid, "cannot find '" + pe->text + "' among the visible columns");
					}
					ns.cols.push_back(*s);
					ns.cols.back().name = pe->text;
				} else {
					throw Error(kErrInvalid, "projection entries must be columns or assignments");
				}
			}
			/* unresolved base columns stay lazily resolvable through the copied entries
			 * (resolve() shares one column slot per base column) */
			sc = ns;
			return pi;
		}
		case RelOp::HashJoin: {
			/* the reference names the join table before translating either side
			 * (relalg_translator.cpp:814): keep its numbering of later aggregations */
			name_counter++;
			/* build side first: its pipeline must run before the probe */
			Scope bs;
			int bi = lower(op->right, bs);
			JoinDesc jd;
			jd.id = (int)out.joins.size();
			jd.join01 = op->join01;
			jd.build_table = out.pipes[bi].table;
			jd.build_rows = rows_bound(out.pipes[bi]);
			Sink sink;
			sink.kind = Sink::JoinBuild;
			sink.join = jd.id;
			int shift = 0;
			for (auto& k : op->right_keys) {
				BExprP e = bind(k, bs, out.pipes[bi]);
				if (e->boolean) {
					throw Error(kErrUnsupported, "join keys must be values");
				}
				sink.keys.push_back(e);
				jd.key_b.push_back(e->b);
				jd.key_shift.push_back(shift);
				shift += bits_for(e->b.hi - e->b.lo + 1);
			}
			jd.key_bits = shift;
			if (jd.key_bits > 62) {
				throw Error(kErrUnsupported, "join key domain needs more than 62 bits");
			}
			jd.key64 = jd.key_bits > 31;
			shift = 0;
			for (auto& pe : op->right_payl) {
				BExprP e = bind(pe, bs, out.pipes[bi]);
				if (e->boolean) {
					throw Error(kErrUnsupported, "join payloads must be values");
				}
				sink.pay.push_back(e);
				jd.pay_b.push_back(e->b);
				jd.pay_shift.push_back(shift);
				shift += bits_for(e->b.hi - e->b.lo + 1);
			}
			jd.pay_bits = shift;
			if (jd.pay_bits > 64) {
				throw Error(kErrUnsupported, "join payload needs more than 64 bits");
			}
			jd.pay64 = jd.pay_bits > 32;
			if (out.pipes[bi].sink.kind != Sink::Emit) {
				throw Error(kErrUnsupported, "the build side of a join must be a scan/select/project/join chain");
			}
			out.pipes[bi].sink = sink;
			out.joins.push_back(jd);

			int pi = lower(op->left, sc);
			Op pr;
			pr.kind = Op::Probe;
			pr.join = jd.id;
			for (auto& k : op->left_keys) {
				BExprP e = bind(k, sc, out.pipes[pi]);
				if (e->boolean) {
					throw Error(kErrUnsupported, "join keys must be values");
				}
				pr.keys.push_back(e);
			}
			pr.npay = (int)jd.pay_b.size();
			const int opi = (int)out.pipes[pi].ops.size();
			out.pipes[pi].ops.push_back(pr);
			/* visible after the join: probe columns, build keys (= probe keys), payloads */
			for (size_t k = 0; k < op->right_keys.size(); k++) {
				if (op->right_keys[k]->kind != RelExpr::ColId) {
					throw Error(kErrUnsupported, "build keys must be column references");
				}
				sc.cols.push_back(ScopeEntry{op->right_keys[k]->text, pr.keys[k], "", ""});
			}
			for (size_t k = 0; k < op->right_payl.size(); k++) {
				if (op->right_payl[k]->kind != RelExpr::ColId) {
					throw Error(kErrUnsupported, "build payloads must be column references");
				}
				auto e = std::make_shared<BExpr>();
				e->kind = BExpr::ProbeOut;
				e->probe = opi;
				e->pidx = (int)k;
				e->b = jd.pay_b[k];
				e->str = sink.pay[k]->str;
				sc.cols.push_back(ScopeEntry{op->right_payl[k]->text, e, "", ""});
			}
			return pi;
		}
		case RelOp::HashAggr:
			return lower_inner_aggregate(op, sc);
		}
		throw Error(kErrInvalid, "bad operator");
	}

	int64_t rows_bound(const Pipeline& p) {
		__int128 r = p.rows;
		for (auto& o : p.ops) {
			if (o.kind == Op::Probe && !out.joins[o.join].join01) {
				r *= std::max<int64_t>(1, out.joins[o.join].build_rows);
			}
		}
		return r > kI64Max ? INT64_MAX : (int64_t)r;
	}

	/* The sink of an aggregation over pipeline pi's rows (visible columns in sc): global,
	 * dense slots or a hash table (relalg_translator.cpp:380-656).  *vis = result columns. */
	/* A sum whose bound leaves int64 (the reference types it i128, typing_pass.cpp:244-259)
	 * becomes sums of bit chunks of its argument that each stay exact in int64: chunks
	 * j < k-1 are the unsigned c-bit fields (v >> j*c) & (2^c - 1), the last is the signed
	 * v >> (k-1)*c, and v is their sum shifted back (two's complement: v == sum over j of
	 * chunk_j << j*c); c leaves room for `rows` additions.  Returns (chunk, shift) pairs. */
	std::vector<std::pair<BExprP, int>> split_wide_sum(const BExprP& v, int64_t rows) {
		const int L = bits_for((__int128)rows + 1);
		const int c = std::max(1, 62 - L);
		for (int k = 2; k <= 64; k++) {
			std::vector<std::pair<BExprP, int>> parts;
			bool fits = true;
			for (int j = 0; j < k; j++) {
				BExprP e = v;
				if (j > 0) {
					e = internal_fun("shr", e, j * c);
				}
				if (j + 1 < k) {
					e = internal_fun("lowbits", e, c);
				}
				const Bounds sb = sum_bounds(e->b, rows);
				fits = fits && sb.lo >= kI64Min && sb.hi <= kI64Max;
				parts.push_back({e, j * c});
			}
			if (fits) {
				return parts;
			}
		}
		throw Error(kErrUnsupported, "sum cannot be split into int64 parts");
	}

	/* shr(x, s) = x >> s (arithmetic: floor(x / 2^s)), lowbits(x, b) = x & (2^b - 1) */
	static BExprP internal_fun(const std::string& fn, const BExprP& x, int amount) {
		auto c = std::make_shared<BExpr>();
		c->kind = BExpr::Const;
		c->cval = amount;
		c->b.lo = c->b.hi = amount;
		auto e = std::make_shared<BExpr>();
		e->kind = BExpr::Fun;
		e->fn = fn;
		e->args = {x, c};
		if (fn == "shr") {
			const __int128 d = (__int128)1 << amount;
			auto floordiv = [&](__int128 a) { return a >= 0 ? a / d : -((-a + d - 1) / d); };
			e->b.lo = floordiv(x->b.lo);
			e->b.hi = floordiv(x->b.hi);
		} else {
			const __int128 m = ((__int128)1 << amount) - 1;
			const bool inside = x->b.lo >= 0 && x->b.hi <= m;
			e->b.lo = inside ? x->b.lo : 0;
			e->b.hi = inside ? x->b.hi : m;
		}
		return e;
	}

	Sink make_agg_sink(const RelOpP& op, Scope& sc, int pi, int* vis, bool allow_wide = false,
		std::vector<OutCol>* outs = nullptr) {
		Pipeline& p = out.pipes[pi];
		const Flavor pf = fl.for_pipe(pi);
		Sink sink;
		const int64_t rows = rows_bound(p);
		std::vector<std::vector<int>> part_shifts; /* per plan aggregate: the shift of each sink part */
		for (auto& k : op->exprs) {
			BExprP e = bind(k, sc, p);
			if (e->boolean) {
				throw Error(kErrUnsupported, "group keys must be values");
			}
			sink.keys.push_back(e);
		}
		for (auto& a : op->aggregates) {
			if (a->kind != RelExpr::Fun || (a->text != "sum" && a->text != "count")) {
				throw Error(kErrUnsupported, "aggregates must be sum(expr) or count()");
			}
			Sink::Agg ag;
			if (a->text == "count") {
				ag.count = true;
				sink.count_idx = (int)sink.aggs.size();
			} else {
				if (a->args.size() != 1) {
					throw Error(kErrInvalid, "sum takes one argument");
				}
				ag.arg = bind(a->args[0], sc, p);
				if (ag.arg->str) {
					throw Error(kErrUnsupported, "sum over a string is not supported");
				}
				if (ag.arg->boolean) {
					throw Error(kErrUnsupported, "sum over a predicate is not supported");
				}
				const Bounds sb = sum_bounds(ag.arg->b, rows);
				if (allow_wide && (sb.lo < kI64Min || sb.hi > kI64Max)) {
					std::vector<int> shifts;
					for (auto& pt : split_wide_sum(ag.arg, rows)) {
						Sink::Agg pa;
						pa.arg = pt.first;
						sink.aggs.push_back(pa);
						shifts.push_back(pt.second);
					}
					part_shifts.push_back(shifts);
					continue;
				}
				check_range(sb, "sum(...) over " + std::to_string(rows) + " rows");
			}
			part_shifts.push_back({0});
			sink.aggs.push_back(ag);
		}
		if (sink.count_idx < 0) {
			Sink::Agg ag;
			ag.count = true;
			ag.visible = false;
			sink.count_idx = (int)sink.aggs.size();
			sink.aggs.push_back(ag);
		}
		if (op->global) {
			sink.kind = Sink::AggGlobal;
			sink.groups_bound = 1;
		} else {
			if (sink.keys.empty()) {
				throw Error(kErrInvalid, "hash aggregation needs keys");
			}
			__int128 domain = 1;
			int shift = 0;
			for (auto& k : sink.keys) {
				const __int128 range = k->b.hi - k->b.lo + 1;
				sink.key_shift.push_back(shift);
				shift += bits_for(range);
				domain *= range;
				if (domain > ((__int128)1 << 100)) {
					domain = (__int128)1 << 100;
				}
			}
			/* mixed-radix strides for the dense slot index (last key fastest) */
			sink.key_radix.assign(sink.keys.size(), 1);
			__int128 stride = 1;
			for (int i = (int)sink.keys.size() - 1; i >= 0; i--) {
				sink.key_radix[i] = stride > kI64Max ? 0 : (int64_t)stride;
				stride *= sink.keys[i]->b.hi - sink.keys[i]->b.lo + 1;
				if (stride > kI64Max) {
					stride = kI64Max;
				}
			}
			sink.key_bits = shift;
			sink.domain = domain;
			__int128 gb = std::min<__int128>(domain, std::max<int64_t>(rows, 1));
			sink.groups_bound = (int64_t)gb;
			const bool dense_ok = domain <= (__int128)pf.dense_limit;
			if (pf.aggr == "dense" && domain > (__int128)(1 << 22)) {
				throw Error(kErrUnsupported, "aggr=dense needs a key domain of at most 2^22 slots");
			}
			if (pf.aggr == "dense" || (pf.aggr == "auto" && dense_ok)) {
				sink.kind = Sink::AggDense;
			} else {
				if (sink.key_bits > 62) {
					throw Error(kErrUnsupported, "group key domain needs more than 62 bits");
				}
				sink.kind = Sink::AggHash;
				pack_aggregates(sink, rows);
			}
		}
		int v = (int)sink.keys.size();
		for (auto& a : sink.aggs) {
			v += a.visible ? 1 : 0;
		}
		*vis = v;
		if (outs) {
			/* the caller's columns: keys, then each plan aggregate over its sink parts */
			outs->clear();
			int phys = 0;
			for (size_t k = 0; k < sink.keys.size(); k++) {
				outs->push_back(OutCol{{{phys++, 0}}, sink.keys[k]->str});
			}
			for (size_t i = 0; i < op->aggregates.size(); i++) {
				OutCol oc;
				for (int sh : part_shifts[i]) {
					oc.parts.push_back({phys++, sh});
				}
				outs->push_back(oc);
			}
		}
		return sink;
	}

	static Bounds sum_bounds(const Bounds& b, int64_t rows) {
		Bounds sb;
		sb.lo = b.lo < 0 ? b.lo * rows : 0;
		sb.hi = b.hi > 0 ? b.hi * rows : 0;
		return sb;
	}

	void aggregate(const RelOpP& op) {
		Scope sc;
		int pi = lower(op->left, sc);
		name_counter += 2;
		int vis = 0;
		out.pipes[pi].sink = make_agg_sink(op, sc, pi, &vis, true, &out.out_cols);
		out.result_pipe = pi;
		out.result_cols = vis;
	}

	/* An aggregation below the root: its rows (keys, then the visible aggregates) go to an
	 * intermediate table named like the reference's re-aggregation table, aggr_ht<N> with
	 * columns key_<i> and aggr_<j> (relalg_translator.cpp:392, :740-760, :776-808), and a new
	 * pipeline scans it. */
	int lower_inner_aggregate(const RelOpP& op, Scope& sc) {
		Scope csc;
		const int pi = lower(op->left, csc);
		name_counter += 2;
		const std::string name = "aggr_ht" + std::to_string(name_counter - 1);
		int vis = 0;
		Sink sink = make_agg_sink(op, csc, pi, &vis);
		const int64_t rows = rows_bound(out.pipes[pi]);
		InterTable it;
		it.name = name;
		it.producer = pi;
		switch (sink.kind) {
		case Sink::AggGlobal: it.cap = 1; break;
		case Sink::AggDense: it.cap = (int64_t)sink.domain; break;
		default: it.cap = std::max<int64_t>(sink.groups_bound, 1); break;
		}
		it.cap = (it.cap + 1) & ~(int64_t)1; /* even: every column starts 16-byte aligned */
		Table t;
		t.name = name;
		t.rows = it.cap;
		for (size_t i = 0; i < sink.keys.size(); i++) {
			Column c;
			c.name = "key_" + std::to_string(i);
			c.type = VC_TYPE_I64;
			c.lo = (int64_t)sink.keys[i]->b.lo;
			c.hi = (int64_t)sink.keys[i]->b.hi;
			c.str = sink.keys[i]->str;
			t.cols.push_back(c);
		}
		int j = 0;
		for (auto& a : sink.aggs) {
			if (!a.visible) {
				continue;
			}
			Column c;
			c.name = "aggr_" + std::to_string(j++);
			c.type = VC_TYPE_I64;
			if (a.count) {
				c.lo = 0;
				c.hi = std::max<int64_t>(rows, 1);
			} else {
				const Bounds sb = sum_bounds(a.arg->b, rows);
				c.lo = (int64_t)sb.lo;
				c.hi = (int64_t)sb.hi;
			}
			t.cols.push_back(c);
		}
		it.cols = t.cols;
		out.pipes[pi].sink = sink;
		out.pipes[pi].out_inter = (int)out.inters.size();
		out.inters.push_back(it);
		inter_tables[name] = t;

		Pipeline np;
		np.id = (int)out.pipes.size();
		np.table = name;
		np.rows = it.cap;
		np.source_inter = (int)out.inters.size() - 1;
		np.sink.kind = Sink::Emit;
		sc.cols.clear();
		for (auto& c : t.cols) {
			sc.cols.push_back(ScopeEntry{name + "." + c.name, nullptr, name, c.name});
		}
		out.pipes.push_back(np);
		return np.id;
	}

	/* First-fit-decreasing packing of the aggregates' bit fields into 64-bit words: the
	 * field of a sum holds sum(value - lo) <= (hi - lo) * rows, a count's holds <= rows. */
	static void pack_aggregates(Sink& sink, int64_t rows) {
		const size_t A = sink.aggs.size();
		sink.agg_word.assign(A, 0);
		sink.agg_shift.assign(A, 0);
		sink.agg_bits.assign(A, 0);
		for (size_t a = 0; a < A; a++) {
			const __int128 r = std::max<int64_t>(rows, 1);
			const __int128 bound = sink.aggs[a].count ? r : (sink.aggs[a].arg->b.hi - sink.aggs[a].arg->b.lo) * r;
			sink.agg_bits[a] = std::max(1, bits_for(bound + 1));
		}
		std::vector<size_t> order(A);
		for (size_t a = 0; a < A; a++) {
			order[a] = a;
		}
		std::stable_sort(order.begin(), order.end(),
			[&](size_t x, size_t y) { return sink.agg_bits[x] > sink.agg_bits[y]; });
		std::vector<int> used;
		for (size_t a : order) {
			size_t w = 0;
			while (w < used.size() && used[w] + sink.agg_bits[a] > 64) {
				w++;
			}
			if (w == used.size()) {
				used.push_back(0);
			}
			sink.agg_word[a] = (int)w;
			sink.agg_shift[a] = used[w];
			used[w] += sink.agg_bits[a];
		}
		sink.nwords = (int)used.size();
	}

	void root(const RelOpP& op) {
		if (op->kind == RelOp::HashAggr) {
			aggregate(op);
			return;
		}
		Scope sc;
		int pi = lower(op, sc);
		Pipeline& p = out.pipes[pi];
		p.sink.kind = Sink::Emit;
		for (auto& s : sc.cols) {
			BExprP e = resolve(s, p);
			if (e->boolean) {
				throw Error(kErrUnsupported, "predicate columns cannot be emitted");
			}
			p.sink.outs.push_back(e);
		}
		p.sink.groups_bound = rows_bound(p);
		out.result_pipe = pi;
		out.result_cols = (int)p.sink.outs.size();
		for (int c = 0; c < out.result_cols; c++) {
			out.out_cols.push_back(OutCol{{{c, 0}}, p.sink.outs[(size_t)c]->str});
		}
	}
};

} // namespace

LoweredPlan lower_plan(const RelOpP& root, std::map<std::string, Table>& tables, const Flavor& fl,
	const StringDict& dict)
{
	Lowerer l(tables, fl, dict);
	l.root(root);
	if (l.out.result_cols == 0) {
		throw Error(kErrInvalid, "the plan produces no columns");
	}
	return l.out;
}

} // namespace vc
