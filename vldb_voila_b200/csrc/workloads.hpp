/*
 * Synthetic workloads for the hot path: table/column generator specs plus the relational
 * plan (as plan text) that runs over them.  They stand in for the reference's TPC-H/SSB
 * setup (bench_tpch.cpp:8-101) and hand-written plans (bench_tpch_rel.cpp), whose data
 * files are not available:
 *
 *   sel_aggr   selection + low-cardinality group-by, TPC-H Q1 shaped (bench_tpch_rel.cpp:26-84)
 *   join_aggr  Join01 hash join + global aggregate, imv1 shaped (bench_tpch_rel.cpp:842-891)
 *   groupby    high-cardinality group-by with Zipf-skewed keys (q18's lineitem group-by)
 *   star       4-dimension probe chain + (year, region) group-by, SSB q4.1 shaped
 *              (db-engine-paradigms/src/benchmarks/sbb/queries/q41.cpp:21-46)
 *   batch      a seeded list of the first three with random sizes, selectivities and skews
 *   bigsum     sums of 64-bit values that leave int64 (128-bit results)
 *   strings    string columns (dictionary codes on the device): contains, string group keys
 *
 * A workload is named by a spec string "<template>:key=value,...", e.g.
 * "join_aggr:build=1500000,probe=6000000,sel=0.2,seed=2".  Header-only C++ so that the
 * engine, its C ABI (vc_workload_describe) and the reference harness share one definition.
 */
#ifndef VOILA_B200_WORKLOADS_HPP
#define VOILA_B200_WORKLOADS_HPP

#include <cmath>
#include <cstdint>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "datagen.h"

namespace vc_workload {

struct Column {
	std::string name;
	vc_gen_spec spec;
	int64_t lo; /* declared value domain: the min/max the plan is typed with */
	int64_t hi;
};

struct Table {
	std::string name;
	int64_t rows;
	std::vector<Column> cols;
};

struct Workload {
	std::string spec;
	std::string tmpl;
	std::vector<Table> tables;
	std::string plan;
	std::string fact_table;      /* the table whose rows are counted as "fact rows" */
	int64_t fact_rows = 0;
	int64_t algo_bytes = 0;      /* bytes a step must read at least (all scanned columns once) */
	int64_t probe_bytes = 0;     /* bytes the dominant (fact) pipeline must read */
};

inline std::map<std::string, std::string> parse_params(const std::string& s, std::string& tmpl)
{
	std::map<std::string, std::string> p;
	auto colon = s.find(':');
	tmpl = s.substr(0, colon);
	if (colon == std::string::npos) {
		return p;
	}
	std::stringstream ss(s.substr(colon + 1));
	std::string item;
	while (std::getline(ss, item, ',')) {
		if (item.empty()) {
			continue;
		}
		auto eq = item.find('=');
		if (eq == std::string::npos) {
			throw std::invalid_argument("workload parameter without '=': " + item);
		}
		p[item.substr(0, eq)] = item.substr(eq + 1);
	}
	return p;
}

inline int64_t param_i(std::map<std::string, std::string>& p, const std::string& k, int64_t def)
{
	auto it = p.find(k);
	if (it == p.end()) {
		return def;
	}
	double v = std::stod(it->second);
	if (v < 0) {
		throw std::invalid_argument("negative workload parameter " + k);
	}
	return (int64_t)std::llround(v);
}

inline double param_f(std::map<std::string, std::string>& p, const std::string& k, double def)
{
	auto it = p.find(k);
	return it == p.end() ? def : std::stod(it->second);
}

inline uint64_t column_seed(uint64_t seed, int table, int col)
{
	return vc_gen_mix64(seed * UINT64_C(1000003) + (uint64_t)table * 131 + (uint64_t)col + 1);
}

/* Builds one column and its declared domain from the generator parameters. */
inline Column make_col(const std::string& name, int type, int kind, int64_t a, int64_t b,
	int64_t rows, uint64_t seed, double s = 0.0, int64_t c = 1)
{
	Column col;
	col.name = name;
	col.spec.kind = kind;
	col.spec.type = type;
	col.spec.a = a;
	col.spec.b = b;
	col.spec.c = c;
	col.spec.s = s;
	col.spec.seed = seed;
	col.spec.n = rows;
	const int64_t last = rows > 0 ? rows - 1 : 0;
	switch (kind) {
	case VC_GEN_UNIFORM: col.lo = a; col.hi = b; break;
	case VC_GEN_SEQ:
	case VC_GEN_PERM: col.lo = a; col.hi = a + last; break;
	case VC_GEN_ZIPF: col.lo = 1; col.hi = b; break;
	case VC_GEN_CHOICE: {
		int64_t lo = 255, hi = 0;
		for (int64_t k = 0; k < b; k++) {
			int64_t v = (a >> (8 * k)) & 0xff;
			lo = v < lo ? v : lo;
			hi = v > hi ? v : hi;
		}
		col.lo = lo;
		col.hi = hi;
		break;
	}
	case VC_GEN_DIV: col.lo = a; col.hi = a + (last * c) / b; break;
	case VC_GEN_MOD: col.lo = a; col.hi = a + (rows < b ? last : b - 1); break;
	case VC_GEN_WORDS: col.lo = 0; col.hi = 0; break; /* strings: the domain is their dictionary codes */
	default: throw std::invalid_argument("bad generator kind");
	}
	return col;
}

inline int64_t pack_chars(const char* s)
{
	int64_t v = 0;
	for (int k = 0; s[k]; k++) {
		v |= (int64_t)(unsigned char)s[k] << (8 * k);
	}
	return v;
}

inline int64_t table_bytes(const Table& t)
{
	int64_t b = 0;
	for (auto& c : t.cols) {
		b += t.rows * vc_gen_type_size(c.spec.type);
	}
	return b;
}

/* first day of the 2,526-day ship-date range, as a Julian day number (1992-01-01) */
static const int64_t kShipDate0 = 2448623;

inline Workload make(const std::string& spec)
{
	Workload w;
	w.spec = spec;
	auto p = parse_params(spec, w.tmpl);
	const uint64_t seed = (uint64_t)param_i(p, "seed", 1);

	if (w.tmpl == "sel_aggr") {
		const int64_t n = param_i(p, "rows", 6000000);
		const double sel = param_f(p, "sel", -1.0);
		const int64_t cut = sel < 0 ? kShipDate0 + 2435
			: kShipDate0 + (int64_t)std::llround(sel * 2526.0) - 1;
		Table t{"lineitem", n, {}};
		t.cols.push_back(make_col("l_quantity", VC_TYPE_I32, VC_GEN_UNIFORM, 1, 50, n, column_seed(seed, 0, 0)));
		t.cols.push_back(make_col("l_extendedprice", VC_TYPE_I64, VC_GEN_UNIFORM, 90000, 10500000, n, column_seed(seed, 0, 1)));
		t.cols.push_back(make_col("l_discount", VC_TYPE_I32, VC_GEN_UNIFORM, 0, 10, n, column_seed(seed, 0, 2)));
		t.cols.push_back(make_col("l_tax", VC_TYPE_I32, VC_GEN_UNIFORM, 0, 8, n, column_seed(seed, 0, 3)));
		t.cols.push_back(make_col("l_returnflag", VC_TYPE_U8, VC_GEN_CHOICE, pack_chars("ANR"), 3, n, column_seed(seed, 0, 4)));
		t.cols.push_back(make_col("l_linestatus", VC_TYPE_U8, VC_GEN_CHOICE, pack_chars("FO"), 2, n, column_seed(seed, 0, 5)));
		t.cols.push_back(make_col("l_shipdate", VC_TYPE_I32, VC_GEN_UNIFORM, kShipDate0, kShipDate0 + 2525, n, column_seed(seed, 0, 6)));
		w.tables.push_back(t);
		std::ostringstream o;
		o << "(aggr hash ((col lineitem.l_returnflag) (col lineitem.l_linestatus))"
		  << " ((fun sum (col lineitem.l_quantity)) (fun sum (col lineitem.l_extendedprice))"
		  << " (fun sum (col disc_price)) (fun sum (col charge)) (fun count))"
		  << " (project ((assign disc_price (fun * (col lineitem.l_extendedprice) (fun - (const 100) (col lineitem.l_discount))))"
		  << " (assign charge (fun * (col disc_price) (fun + (const 100) (col lineitem.l_tax))))"
		  << " (col lineitem.l_quantity) (col lineitem.l_extendedprice) (col lineitem.l_returnflag) (col lineitem.l_linestatus))"
		  << " (select (fun <= (col lineitem.l_shipdate) (const " << cut << "))"
		  << " (scan lineitem (l_shipdate l_returnflag l_linestatus l_extendedprice l_quantity l_discount l_tax)))))";
		w.plan = o.str();
		w.fact_table = "lineitem";
		w.fact_rows = n;
		w.algo_bytes = table_bytes(t);
		w.probe_bytes = w.algo_bytes;
	} else if (w.tmpl == "join_aggr") {
		const int64_t nb = param_i(p, "build", 1500000);
		const int64_t np = param_i(p, "probe", 6000000);
		const double sel = param_f(p, "sel", 0.2);
		const int64_t thr = (int64_t)std::llround(sel * 10000.0);
		Table b{"orders", nb, {}};
		b.cols.push_back(make_col("o_orderkey", VC_TYPE_I32, VC_GEN_PERM, 1, 0, nb, column_seed(seed, 0, 0)));
		b.cols.push_back(make_col("o_attr", VC_TYPE_I32, VC_GEN_UNIFORM, 0, 9999, nb, column_seed(seed, 0, 1)));
		Table f{"lineitem", np, {}};
		f.cols.push_back(make_col("l_orderkey", VC_TYPE_I32, VC_GEN_UNIFORM, 1, nb > 0 ? nb : 1, np, column_seed(seed, 1, 0)));
		f.cols.push_back(make_col("l_val", VC_TYPE_I64, VC_GEN_UNIFORM, 1, 1000000, np, column_seed(seed, 1, 1)));
		w.tables.push_back(b);
		w.tables.push_back(f);
		std::ostringstream o;
		o << "(aggr global () ((fun sum (col lineitem.l_val)) (fun count))"
		  << " (join join01 ((col lineitem.l_orderkey)) ()"
		  << " (scan lineitem (l_orderkey l_val))"
		  << " ((col orders.o_orderkey)) ()"
		  << " (select (fun < (col orders.o_attr) (const " << thr << ")) (scan orders (o_orderkey o_attr)))))";
		w.plan = o.str();
		w.fact_table = "lineitem";
		w.fact_rows = np;
		w.algo_bytes = table_bytes(b) + table_bytes(f);
		w.probe_bytes = table_bytes(f);
	} else if (w.tmpl == "groupby") {
		const int64_t n = param_i(p, "rows", 6000000);
		const int64_t keys = param_i(p, "keys", 1500000);
		const double s = param_f(p, "zipf", 0.0);
		if (keys < 1) {
			throw std::invalid_argument("groupby needs keys >= 1");
		}
		Table t{"lineitem", n, {}};
		t.cols.push_back(make_col("l_orderkey", VC_TYPE_I32, VC_GEN_ZIPF, 1, keys, n, column_seed(seed, 0, 0), s));
		t.cols.push_back(make_col("l_extendedprice", VC_TYPE_I64, VC_GEN_UNIFORM, 1, 1000000, n, column_seed(seed, 0, 1)));
		t.cols.push_back(make_col("l_quantity", VC_TYPE_I32, VC_GEN_UNIFORM, 1, 50, n, column_seed(seed, 0, 2)));
		w.tables.push_back(t);
		w.plan = "(aggr hash ((col lineitem.l_orderkey))"
			" ((fun sum (col lineitem.l_extendedprice)) (fun sum (col lineitem.l_quantity)) (fun count))"
			" (scan lineitem (l_orderkey l_extendedprice l_quantity)))";
		w.fact_table = "lineitem";
		w.fact_rows = n;
		w.algo_bytes = table_bytes(t);
		w.probe_bytes = w.algo_bytes;
	} else if (w.tmpl == "star") {
		const int64_t n = param_i(p, "rows", 60000000);
		const int64_t nd = param_i(p, "dates", 2556);
		const int64_t nc = param_i(p, "custs", 300000);
		const int64_t ns = param_i(p, "supps", 20000);
		const int64_t np = param_i(p, "parts", 1400000);
		if (nd < 1 || nc < 1 || ns < 1 || np < 1) {
			throw std::invalid_argument("star needs non-empty dimensions");
		}
		Table d{"date", nd, {}};
		d.cols.push_back(make_col("d_datekey", VC_TYPE_I32, VC_GEN_SEQ, 1, 0, nd, column_seed(seed, 0, 0)));
		d.cols.push_back(make_col("d_year", VC_TYPE_I16, VC_GEN_DIV, 1992, nd, nd, column_seed(seed, 0, 1), 0.0, 7));
		d.cols.push_back(make_col("d_weekday", VC_TYPE_U8, VC_GEN_MOD, 0, 7, nd, column_seed(seed, 0, 2)));
		Table c{"customer", nc, {}};
		c.cols.push_back(make_col("c_custkey", VC_TYPE_I32, VC_GEN_SEQ, 1, 0, nc, column_seed(seed, 1, 0)));
		c.cols.push_back(make_col("c_region", VC_TYPE_U8, VC_GEN_UNIFORM, 0, 4, nc, column_seed(seed, 1, 1)));
		c.cols.push_back(make_col("c_mktsegment", VC_TYPE_U8, VC_GEN_UNIFORM, 0, 4, nc, column_seed(seed, 1, 2)));
		Table s{"supplier", ns, {}};
		s.cols.push_back(make_col("s_suppkey", VC_TYPE_I32, VC_GEN_SEQ, 1, 0, ns, column_seed(seed, 2, 0)));
		Table pt{"part", np, {}};
		pt.cols.push_back(make_col("p_partkey", VC_TYPE_I32, VC_GEN_SEQ, 1, 0, np, column_seed(seed, 3, 0)));
		pt.cols.push_back(make_col("p_category", VC_TYPE_U8, VC_GEN_UNIFORM, 0, 24, np, column_seed(seed, 3, 1)));
		Table f{"lineorder", n, {}};
		f.cols.push_back(make_col("lo_orderdate", VC_TYPE_I32, VC_GEN_UNIFORM, 1, nd, n, column_seed(seed, 4, 0)));
		f.cols.push_back(make_col("lo_custkey", VC_TYPE_I32, VC_GEN_UNIFORM, 1, nc, n, column_seed(seed, 4, 1)));
		f.cols.push_back(make_col("lo_suppkey", VC_TYPE_I32, VC_GEN_UNIFORM, 1, ns, n, column_seed(seed, 4, 2)));
		f.cols.push_back(make_col("lo_partkey", VC_TYPE_I32, VC_GEN_UNIFORM, 1, np, n, column_seed(seed, 4, 3)));
		f.cols.push_back(make_col("lo_revenue", VC_TYPE_I64, VC_GEN_UNIFORM, 1, 10000000, n, column_seed(seed, 4, 4)));
		f.cols.push_back(make_col("lo_supplycost", VC_TYPE_I64, VC_GEN_UNIFORM, 1, 100000, n, column_seed(seed, 4, 5)));
		w.tables = {d, c, s, pt, f};
		w.plan =
			"(aggr hash ((col date.d_year) (col customer.c_region)) ((fun sum (col profit)))"
			" (project ((assign profit (fun - (col lineorder.lo_revenue) (col lineorder.lo_supplycost)))"
			" (col date.d_year) (col customer.c_region))"
			" (join join01 ((col lineorder.lo_suppkey)) ()"
			"  (join join01 ((col lineorder.lo_custkey)) ()"
			"   (join join01 ((col lineorder.lo_orderdate)) ()"
			"    (join join01 ((col lineorder.lo_partkey)) ()"
			"     (scan lineorder (lo_orderdate lo_custkey lo_suppkey lo_partkey lo_revenue lo_supplycost))"
			"     ((col part.p_partkey)) ()"
			"     (select (fun = (col part.p_category) (const 7)) (scan part (p_partkey p_category))))"
			"    ((col date.d_datekey)) ((col date.d_year))"
			"    (select (fun = (col date.d_weekday) (const 3)) (scan date (d_datekey d_year d_weekday))))"
			"   ((col customer.c_custkey)) ((col customer.c_region))"
			"   (select (fun = (col customer.c_mktsegment) (const 1)) (scan customer (c_custkey c_region c_mktsegment))))"
			"  ((col supplier.s_suppkey)) ()"
			"  (scan supplier (s_suppkey)))))";
		w.fact_table = "lineorder";
		w.fact_rows = n;
		w.algo_bytes = table_bytes(d) + table_bytes(c) + table_bytes(s) + table_bytes(pt) + table_bytes(f);
		w.probe_bytes = table_bytes(f);
	} else if (w.tmpl == "strings") {
		/* string columns: part names of three words from a 24-word list, one-word brands from
		 * the first six; a fact table of part references (TPC-H q9's `contains` shape) */
		const int64_t n = param_i(p, "rows", 200000);
		const int64_t np = param_i(p, "parts", 20000);
		if (np < 1) {
			throw std::invalid_argument("strings needs parts >= 1");
		}
		Table pt{"part", np, {}};
		pt.cols.push_back(make_col("p_partkey", VC_TYPE_I32, VC_GEN_SEQ, 1, 0, np, column_seed(seed, 0, 0)));
		pt.cols.push_back(make_col("p_name", VC_TYPE_STR, VC_GEN_WORDS, 3, 24, np, column_seed(seed, 0, 1)));
		pt.cols.push_back(make_col("p_brand", VC_TYPE_STR, VC_GEN_WORDS, 1, 6, np, column_seed(seed, 0, 2)));
		Table f{"lineitem", n, {}};
		f.cols.push_back(make_col("l_partkey", VC_TYPE_I32, VC_GEN_UNIFORM, 1, np, n, column_seed(seed, 1, 0)));
		f.cols.push_back(make_col("l_extendedprice", VC_TYPE_I64, VC_GEN_UNIFORM, 1, 1000000, n, column_seed(seed, 1, 1)));
		w.tables = {pt, f};
		w.plan = "(aggr hash ((col part.p_brand)) ((fun sum (col lineitem.l_extendedprice)) (fun count))"
			" (join join01 ((col lineitem.l_partkey)) () (scan lineitem (l_partkey l_extendedprice))"
			" ((col part.p_partkey)) ((col part.p_brand))"
			" (select (fun contains (col part.p_name) (const green)) (scan part (p_partkey p_name p_brand)))))";
		w.fact_table = "lineitem";
		w.fact_rows = n;
		w.algo_bytes = table_bytes(pt) + table_bytes(f);
		w.probe_bytes = table_bytes(f);
	} else if (w.tmpl == "bigsum") {
		/* sums whose bound leaves int64 (the reference types them i128): 64-bit values up to
		 * +-2e15 (exact in a double, where the reference's min/max typing stays exact) grouped
		 * by a 2-bit key; 10,000 of them per group already sum past 2^63 */
		const int64_t n = param_i(p, "rows", 40000);
		Table t{"fact", n, {}};
		t.cols.push_back(make_col("g", VC_TYPE_U8, VC_GEN_UNIFORM, 0, 3, n, column_seed(seed, 0, 0)));
		t.cols.push_back(make_col("v", VC_TYPE_I64, VC_GEN_UNIFORM, -2000000000000000ll, 2000000000000000ll, n,
			column_seed(seed, 0, 1)));
		t.cols.push_back(make_col("w", VC_TYPE_I64, VC_GEN_UNIFORM, 0, 2000000000000000ll, n, column_seed(seed, 0, 2)));
		w.tables.push_back(t);
		w.plan = "(aggr hash ((col fact.g)) ((fun sum (col fact.v)) (fun sum (col fact.w)) (fun count))"
			" (scan fact (g v w)))";
		w.fact_table = "fact";
		w.fact_rows = n;
		w.algo_bytes = table_bytes(t);
		w.probe_bytes = w.algo_bytes;
	} else {
		throw std::invalid_argument("unknown workload template '" + w.tmpl + "'");
	}
	return w;
}

/*
 * The mixed batch: `count` pipelines drawn by `seed` from sel_aggr / join_aggr / groupby,
 * fact sizes log-uniform over [min_rows, max_rows], selectivities uniform over [1 %, 100 %],
 * Zipf exponents uniform over [0, 1.25].  Returns one workload spec string per pipeline.
 */
inline std::vector<std::string> make_batch(int count, uint64_t seed, int64_t min_rows, int64_t max_rows)
{
	std::vector<std::string> out;
	for (int i = 0; i < count; i++) {
		auto u = [&](int k) {
			return (double)(vc_gen_bits(seed * 7919 + 17, (uint64_t)i * 8 + k) >> 11) * (1.0 / 9007199254740992.0);
		};
		const int tmpl = (int)(u(0) * 3.0);
		const double lr = std::log((double)min_rows) + u(1) * (std::log((double)max_rows) - std::log((double)min_rows));
		const int64_t rows = (int64_t)std::llround(std::exp(lr));
		const double sel = 0.01 + u(2) * 0.99;
		const double zipf = u(3) * 1.25;
		const uint64_t pseed = seed * 1000 + (uint64_t)i + 1;
		std::ostringstream o;
		o.precision(6);
		if (tmpl == 0) {
			o << "sel_aggr:rows=" << rows << ",sel=" << sel << ",seed=" << pseed;
		} else if (tmpl == 1) {
			int64_t build = rows / 4 > 1 ? rows / 4 : 1;
			o << "join_aggr:build=" << build << ",probe=" << rows << ",sel=" << sel << ",seed=" << pseed;
		} else {
			int64_t keys = rows / 4 > 1 ? rows / 4 : 1;
			if (keys > 1500000) {
				keys = 1500000;
			}
			o << "groupby:rows=" << rows << ",keys=" << keys << ",zipf=" << zipf << ",seed=" << pseed;
		}
		out.push_back(o.str());
	}
	return out;
}

/* Line-oriented text form of a workload, parsed by the Python side. */
inline std::string describe(const Workload& w)
{
	std::ostringstream o;
	o.precision(17);
	o << "workload " << w.spec << "\n";
	o << "template " << w.tmpl << "\n";
	o << "fact " << w.fact_table << " " << w.fact_rows << "\n";
	o << "bytes " << w.algo_bytes << " " << w.probe_bytes << "\n";
	for (auto& t : w.tables) {
		o << "table " << t.name << " " << t.rows << "\n";
		for (auto& c : t.cols) {
			o << "column " << t.name << " " << c.name << " " << c.spec.type << " " << c.spec.kind << " "
			  << c.spec.a << " " << c.spec.b << " " << c.spec.c << " " << c.spec.s << " " << c.spec.seed << " "
			  << c.spec.n << " " << c.lo << " " << c.hi << "\n";
		}
	}
	o << "plan " << w.plan << "\n";
	return o.str();
}

} // namespace vc_workload

#endif
