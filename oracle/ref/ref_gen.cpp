/*
 * Test infrastructure: generates and compiles one of the reference's query libraries.
 *
 * Runs the reference's own front end and code generators -- RelOpTranslator and the
 * HyperCodegen / VectorCodegen selected in Compiler::_generate (compiler.cpp:343-385) -- on
 * a plan given as plan text over a synthetic workload, then compiles the emitted C++ the
 * way Compiler::call_cxx_compiler does (compiler.cpp:19-57), with the flags passed in
 * --cxx.  The result exports voila_query_new/run/reset/free (codegen.cpp:371-392) and is
 * independent of the table sizes: code generation only reads each column's declared
 * min/max (codegen.cpp:11-19).
 *
 * usage: ref_gen --workload SPEC --flavor hyper|vectorwise|cuda --out LIB.so --cxx "g++ ..."
 *                [--plan PLAN-TEXT] [--keep-src FILE] [--link "LDFLAGS"] [--cuda-flavor "cuda(...)"]
 *
 * --flavor cuda plays the part of a Flavor::Cuda case in Compiler::_generate: the plan goes
 * through the reference's relalg tree, is printed back as plan text (cuda_flavor.hpp) and
 * becomes the generated library's constant; the library is the fixed glue (cuda_glue.inc)
 * over libvoila_cuda.so, linked with --link.
 */
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <unistd.h>

#include "common/runtime/Database.hpp"
#include "compiler.hpp"
#include "cuda_flavor.hpp"
#include "ref_plans.hpp"
#include "runtime_framework.hpp"

int main(int argc, char** argv)
{
	std::string spec, flavor = "hyper", out, cxx, plan, keep_src, link, cuda_flavor;
	for (int i = 1; i + 1 < argc; i += 2) {
		std::string k = argv[i];
		if (k == "--workload") spec = argv[i + 1];
		else if (k == "--flavor") flavor = argv[i + 1];
		else if (k == "--out") out = argv[i + 1];
		else if (k == "--cxx") cxx = argv[i + 1];
		else if (k == "--plan") plan = argv[i + 1];
		else if (k == "--keep-src") keep_src = argv[i + 1];
		else if (k == "--link") link = argv[i + 1];
		else if (k == "--cuda-flavor") cuda_flavor = argv[i + 1];
		else {
			std::cerr << "ref_gen: unknown option " << k << std::endl;
			return 2;
		}
	}
	if (spec.empty() || out.empty() || cxx.empty()) {
		std::cerr << "ref_gen: --workload, --out and --cxx are required" << std::endl;
		return 2;
	}
	try {
		auto w = vc_workload::make(spec);
		if (!plan.empty()) {
			w.plan = plan;
		}
		if (flavor == "cuda") {
			auto root = ref_harness::to_ref_op(vc_sexpr::parse(w.plan));
			const std::string src_name = out + ".glue.cpp";
			{
				std::ofstream f(src_name);
				f << voila_cuda_flavor::glue_source(voila_cuda_flavor::plan_text(*root), cuda_flavor);
			}
			std::ostringstream cmd;
			cmd << cxx << " -shared -fPIC " << src_name << " -o " << out << " " << link;
			const int rc = std::system(cmd.str().c_str());
			if (!keep_src.empty()) {
				std::ifstream in(src_name);
				std::ofstream o(keep_src);
				o << in.rdbuf();
			}
			std::remove(src_name.c_str());
			if (rc != 0) {
				std::cerr << "ref_gen: compiler failed: " << cmd.str() << std::endl;
				return 1;
			}
			return 0;
		}
		runtime::Database db;
		ref_harness::load_workload(db, w, 64, 1);

		QueryConfig qconf(db);
		qconf.num_threads = 1;
		if (flavor == "hyper") {
			qconf.flavor = QueryConfig::Flavor::Hyper;
		} else if (flavor == "vectorwise" || flavor == "vector") {
			qconf.flavor = QueryConfig::Flavor::Vectorwise;
		} else {
			std::cerr << "ref_gen: unsupported flavor " << flavor << std::endl;
			return 2;
		}
		BenchmarkQuery bq;
		bq.root = ref_harness::to_ref_op(vc_sexpr::parse(w.plan));

		const std::string postfix = "_refgen_" + std::to_string(getpid());
		Compiler compiler(0, postfix);
		std::stringstream src;
		compiler._generate(qconf, bq, src);

		std::ostringstream cmd;
		cmd << cxx << " -shared -fPIC " << compiler.tmp_fname << " -o " << out;
		int rc = std::system(cmd.str().c_str());
		if (!keep_src.empty()) {
			std::ifstream in(compiler.tmp_fname);
			std::ofstream o(keep_src);
			o << in.rdbuf();
		}
		std::remove(compiler.tmp_fname.c_str());
		if (rc != 0) {
			std::cerr << "ref_gen: compiler failed: " << cmd.str() << std::endl;
			return 1;
		}
	} catch (const std::exception& e) {
		std::cerr << "ref_gen: " << e.what() << std::endl;
		return 1;
	}
	return 0;
}
