/*
 * Test infrastructure (see ref_plans.hpp): plan-text -> reference relalg, and the
 * synthetic workload loader for the reference's runtime::Database.
 */
#include "ref_plans.hpp"

#include <cstring>
#include <stdexcept>
#include <thread>

#include "common/runtime/Database.hpp"
#include "common/runtime/Types.hpp"
#include "common/algebra/Types.hpp"

using vc_sexpr::Node;

namespace ref_harness {

static std::vector<std::shared_ptr<relalg::RelExpr>> expr_list(const Node& n)
{
	std::vector<std::shared_ptr<relalg::RelExpr>> r;
	if (n.atom) {
		throw std::invalid_argument("plan: expected an expression list");
	}
	for (auto& k : n.kids) {
		r.push_back(to_ref_expr(k));
	}
	return r;
}

std::shared_ptr<relalg::RelExpr> to_ref_expr(const Node& n)
{
	const std::string& h = n.head();
	if (h == "const") {
		return std::make_shared<relalg::Const>(n.atom_text(1));
	}
	if (h == "col") {
		return std::make_shared<relalg::ColId>(n.atom_text(1));
	}
	if (h == "assign") {
		return std::make_shared<relalg::Assign>(n.atom_text(1), to_ref_expr(n.at(2)));
	}
	if (h == "fun") {
		std::vector<std::shared_ptr<relalg::RelExpr>> args;
		for (size_t i = 2; i < n.kids.size(); i++) {
			args.push_back(to_ref_expr(n.kids[i]));
		}
		return std::make_shared<relalg::Fun>(n.atom_text(1), args);
	}
	throw std::invalid_argument("plan: unknown expression '" + h + "'");
}

std::shared_ptr<relalg::RelOp> to_ref_op(const Node& n)
{
	const std::string& h = n.head();
	if (h == "scan") {
		std::vector<std::string> cols;
		for (auto& c : n.at(2).kids) {
			cols.push_back(c.text);
		}
		return std::make_shared<relalg::Scan>(n.atom_text(1), relalg::RelExpr::from_column_names(cols));
	}
	if (h == "select") {
		return std::make_shared<relalg::Select>(to_ref_op(n.at(2)), to_ref_expr(n.at(1)));
	}
	if (h == "project") {
		return std::make_shared<relalg::Project>(to_ref_op(n.at(2)), expr_list(n.at(1)));
	}
	if (h == "aggr") {
		const std::string& v = n.atom_text(1);
		auto variant = v == "global" ? relalg::HashAggr::Variant::Global : relalg::HashAggr::Variant::Hash;
		return std::make_shared<relalg::HashAggr>(variant, to_ref_op(n.at(4)), expr_list(n.at(2)),
			expr_list(n.at(3)));
	}
	if (h == "join") {
		const std::string& v = n.atom_text(1);
		auto variant = v == "joinN" ? relalg::HashJoin::Variant::JoinN : relalg::HashJoin::Variant::Join01;
		return std::make_shared<relalg::HashJoin>(variant,
			to_ref_op(n.at(4)), expr_list(n.at(2)), expr_list(n.at(3)),
			to_ref_op(n.at(7)), expr_list(n.at(5)), expr_list(n.at(6)));
	}
	throw std::invalid_argument("plan: unknown operator '" + h + "'");
}

template <typename T>
static void fill(runtime::Attribute& attr, const vc_workload::Column& c, int64_t rows,
	const std::vector<double>& cdf, int threads)
{
	std::vector<T> v((size_t)rows);
	const double* z = cdf.empty() ? nullptr : cdf.data();
	std::vector<std::thread> ws;
	for (int t = 0; t < threads; t++) {
		ws.emplace_back([&, t]() {
			int64_t b = rows * t / threads, e = rows * (t + 1) / threads;
			for (int64_t i = b; i < e; i++) {
				v[(size_t)i] = (T)vc_gen_value(&c.spec, z, i);
			}
		});
	}
	for (auto& w : ws) {
		w.join();
	}
	attr = std::move(v);
}

/* A string column as the reference's varchar attribute: rows of a length byte and
 * VC_GEN_STR_WIDTH - 1 characters (the layout varchar(data, idx, max_len) reads,
 * runtime.hpp:192-204), the varchar views in attr.varchar_data that base-table scans use
 * (runtime_struct.cpp:837-839), and MinMaxInfo with kVariableSize and max_len. */
struct StrRow {
	uint8_t len;
	char chars[VC_GEN_STR_WIDTH - 1];
};

static void load_strings(runtime::Relation& rel, const vc_workload::Column& c, int64_t rows)
{
	std::vector<StrRow> v((size_t)rows);
	char buf[VC_GEN_STR_WIDTH];
	for (int64_t i = 0; i < rows; i++) {
		const int n = vc_gen_string(&c.spec, i, buf);
		StrRow& r = v[(size_t)i];
		std::memset(&r, 0, sizeof(r));
		r.len = (uint8_t)n;
		std::memcpy(r.chars, buf, (size_t)n);
	}
	auto& attr = rel.insert(c.name, std::unique_ptr<algebra::Type>(new algebra::Varchar(VC_GEN_STR_WIDTH - 1)));
	/* through the typed view: Attribute::operator= sizes its buffer for pointer-sized elements */
	auto& vec = attr.typedAccessForChange<StrRow>();
	vec.reset((size_t)rows);
	for (auto& r : v) {
		vec.push_back(r);
	}
	attr.varchar_data.reserve((size_t)rows);
	for (int64_t i = 0; i < rows; i++) {
		attr.varchar_data.emplace_back(varchar(attr.data(), (size_t)i, VC_GEN_STR_WIDTH - 1));
	}
	attr.minmax = new MinMaxInfo();
	attr.minmax->lo = 0;
	attr.minmax->hi = 0;
	attr.minmax->max_len = VC_GEN_STR_WIDTH - 1;
	attr.minmax->flags |= MinMaxInfo::kVariableSize;
}

/* FNV-1a (64-bit) of a string: a string column's contribution to the data checksum */
static int64_t fnv1a(const char* s, size_t n)
{
	uint64_t h = UINT64_C(0xcbf29ce484222325);
	for (size_t i = 0; i < n; i++) {
		h ^= (unsigned char)s[i];
		h *= UINT64_C(0x100000001b3);
	}
	return (int64_t)h;
}

size_t load_workload(runtime::Database& db, const vc_workload::Workload& w, int64_t max_rows, int threads)
{
	size_t values = 0;
	if (threads < 1) {
		threads = 1;
	}
	for (auto& t : w.tables) {
		int64_t rows = t.rows;
		if (max_rows >= 0 && rows > max_rows) {
			rows = max_rows;
		}
		auto& rel = db[t.name];
		rel.name = t.name;
		rel.nrTuples = (size_t)rows;
		for (auto& c : t.cols) {
			std::vector<double> cdf;
			if (c.spec.kind == VC_GEN_ZIPF && c.spec.s != 0.0) {
				cdf.resize((size_t)c.spec.b);
				vc_gen_build_zipf_cdf(c.spec.s, c.spec.b, cdf.data());
			}
			if (c.spec.type == VC_TYPE_STR) {
				load_strings(rel, c, rows);
				values += (size_t)rows;
				continue;
			}
			std::unique_ptr<algebra::Type> type;
			switch (c.spec.type) {
			case VC_TYPE_U8: type.reset(new algebra::Char(1)); break;
			case VC_TYPE_I64: type.reset(new algebra::BigInt()); break;
			/* the reference's Database has no 16-bit attribute type: i16 columns are
			 * stored as Integer (i32) with identical values */
			default: type.reset(new algebra::Integer()); break;
			}
			auto& attr = rel.insert(c.name, std::move(type));
			switch (c.spec.type) {
			case VC_TYPE_U8: fill<uint8_t>(attr, c, rows, cdf, threads); break;
			case VC_TYPE_I64: fill<int64_t>(attr, c, rows, cdf, threads); break;
			default: fill<int32_t>(attr, c, rows, cdf, threads); break;
			}
			attr.minmax = new MinMaxInfo();
			attr.minmax->lo = (double)c.lo;
			attr.minmax->hi = (double)c.hi;
			values += (size_t)rows;
		}
	}
	return values;
}

uint64_t data_checksum(runtime::Database& db, const vc_workload::Workload& w)
{
	uint64_t sum = 0;
	int ti = 0;
	for (auto& t : w.tables) {
		auto& rel = db[t.name];
		int ci = 0;
		for (auto& c : t.cols) {
			auto& attr = rel[c.name];
			for (size_t i = 0; i < rel.nrTuples; i++) {
				int64_t v;
				switch (c.spec.type) {
				case VC_TYPE_STR: v = fnv1a(attr.varchar_data[i].arr, attr.varchar_data[i].len); break;
				case VC_TYPE_U8: v = ((uint8_t*)attr.data())[i]; break;
				case VC_TYPE_I64: v = ((int64_t*)attr.data())[i]; break;
				default: v = ((int32_t*)attr.data())[i]; break;
				}
				sum += vc_gen_mix64((uint64_t)v * 31 + (uint64_t)i * 1000003 + (uint64_t)ti * 131 + (uint64_t)ci);
			}
			ci++;
		}
		ti++;
	}
	return sum;
}

} // namespace ref_harness
