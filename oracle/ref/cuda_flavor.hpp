/*
 * The reference-side binding of the CUDA flavor: what a `Flavor::Cuda` case of the
 * reference's Compiler::_generate (compiler.cpp:343-385) emits instead of pipeline code.
 *
 *   plan_text(root)        the reference's own relalg tree (relalg.hpp:12-178) as the plan
 *                          text libvoila_cuda.so takes (a RelOpVisitor/RelExprVisitor pass)
 *   glue_source(plan, fl)  the generated library's C++ source: the plan and flavor as two
 *                          constants, then cuda_glue.inc, which implements the generated-
 *                          library ABI voila_query_new/run/reset/free (codegen.cpp:371-392)
 *                          on top of libvoila_cuda.so
 *
 * The library is compiled like any generated query (call_cxx_compiler, compiler.cpp:19-57)
 * plus -lvoila_cuda, and Compiler::_run drives it unchanged.  Here ref_gen --flavor cuda
 * builds it and ref_run drives it; the GPU tests compare its rows with the golden outputs of
 * the reference's hyper and vectorwise flavors.
 */
#ifndef VOILA_ORACLE_CUDA_FLAVOR_HPP
#define VOILA_ORACLE_CUDA_FLAVOR_HPP

#include <sstream>
#include <string>

#include "relalg.hpp"

namespace voila_cuda_flavor {

struct PlanText : relalg::RelOpVisitor, relalg::RelExprVisitor {
	std::ostringstream o;

	void list(const std::vector<std::shared_ptr<relalg::RelExpr>>& v) {
		o << "(";
		for (size_t i = 0; i < v.size(); i++) {
			o << (i ? " " : "");
			v[i]->accept(*this);
		}
		o << ")";
	}
	void visit(relalg::Const& c) override { o << "(const " << c.val << ")"; }
	void visit(relalg::ColId& c) override { o << "(col " << c.id << ")"; }
	void visit(relalg::Fun& f) override {
		o << "(fun " << f.name;
		for (auto& a : f.args) {
			o << " ";
			a->accept(*this);
		}
		o << ")";
	}
	void visit(relalg::Assign& a) override {
		o << "(assign " << a.name << " ";
		a.expr->accept(*this);
		o << ")";
	}
	void visit(relalg::Scan& s) override {
		o << "(scan " << s.table << " (";
		for (size_t i = 0; i < s.columns.size(); i++) {
			/* the reference's Scan holds ColIds of bare column names */
			o << (i ? " " : "") << static_cast<relalg::ColId*>(s.columns[i].get())->id;
		}
		o << "))";
	}
	void visit(relalg::Select& s) override {
		o << "(select ";
		s.predicate->accept(*this);
		o << " ";
		s.left->accept(*this);
		o << ")";
	}
	void visit(relalg::Project& p) override {
		o << "(project ";
		list(p.projections);
		o << " ";
		p.left->accept(*this);
		o << ")";
	}
	void visit(relalg::HashAggr& a) override {
		o << "(aggr " << (a.variant == relalg::HashAggr::Global ? "global " : "hash ");
		list(a.keys);
		o << " ";
		list(a.aggregates);
		o << " ";
		a.left->accept(*this);
		o << ")";
	}
	void visit(relalg::HashJoin& j) override {
		o << "(join " << (j.variant == relalg::HashJoin::Join01 ? "join01 " : "joinN ");
		list(j.left_keys);
		o << " ";
		list(j.left_payl);
		o << " ";
		j.left->accept(*this);
		o << " ";
		list(j.right_keys);
		o << " ";
		list(j.right_payl);
		o << " ";
		j.right->accept(*this);
		o << ")";
	}
};

inline std::string plan_text(relalg::RelOp& root)
{
	PlanText pt;
	root.accept(pt);
	return pt.o.str();
}

/* Source of the generated library: constants, then the fixed glue (cuda_glue.inc). */
inline std::string glue_source(const std::string& plan, const std::string& flavor)
{
	std::ostringstream s;
	s << "/* generated for the CUDA flavor */\n";
	s << "static const char* kPlan = R\"VCPLAN(" << plan << ")VCPLAN\";\n";
	s << "static const char* kFlavor = R\"VCPLAN(" << flavor << ")VCPLAN\";\n";
	s << "#include \"cuda_glue.inc\"\n";
	return s.str();
}

} // namespace voila_cuda_flavor

#endif
