/*
 * Test infrastructure: turns plan text (vldb_voila_b200/csrc/sexpr.hpp) into the
 * reference's own relalg tree (relalg.hpp:12-178), so that one plan drives both the
 * reference's hyper/vectorwise flavors and the CUDA engine.  Also loads a synthetic
 * workload (vldb_voila_b200/csrc/workloads.hpp) into the reference's runtime::Database
 * (db-engine-paradigms/include/common/runtime/Database.hpp:28-75), setting each
 * attribute's MinMaxInfo, which the reference's codegen reads to type columns
 * (codegen.cpp:11-19).
 */
#ifndef VOILA_ORACLE_REF_PLANS_HPP
#define VOILA_ORACLE_REF_PLANS_HPP

#include <memory>
#include <string>
#include <vector>

#include "relalg.hpp"
#include "sexpr.hpp"
#include "workloads.hpp"

namespace runtime {
class Database;
}

namespace ref_harness {

std::shared_ptr<relalg::RelExpr> to_ref_expr(const vc_sexpr::Node& n);
std::shared_ptr<relalg::RelOp> to_ref_op(const vc_sexpr::Node& n);

/* Fills `db` with the workload's tables.  `max_rows` < 0 loads every row; otherwise each
 * table is cut to at most max_rows rows (enough for code generation, which only needs the
 * declared min/max).  Returns the total number of loaded values. */
size_t load_workload(runtime::Database& db, const vc_workload::Workload& w, int64_t max_rows,
	int threads);

/* order-insensitive 64-bit checksum of all loaded columns (sum of mixed (table, col, row, value)) */
uint64_t data_checksum(runtime::Database& db, const vc_workload::Workload& w);

} // namespace ref_harness

#endif
