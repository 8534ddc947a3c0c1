/*
 * Test infrastructure: runs one of the reference's compiled query libraries (see ref_gen)
 * on a synthetic workload, the way Compiler::_run does (compiler.cpp:465-598): dlopen, dlsym
 * of the voila_query_* ABI, qnew, then per hot repetition qreset + a timed qrun.
 *
 * usage: ref_run --workload SPEC --lib LIB.so --flavor hyper|vectorwise|cuda
 *                [--threads N] [--reps R] [--result FILE] [--no-result 1] [--checksum 1]
 *                [--max-rows N] [--vector-size N] [--morsel-size N]
 *
 * Prints one JSON line: {"times_ms": [...], "threads": N, "rows": R, "checksum": C}.
 * With --result, the QueryResult text of the last repetition (runtime_framework.cpp:77-111)
 * is written to FILE.
 */
#include <chrono>
#include <cstdio>
#include <dlfcn.h>
#include <fstream>
#include <iostream>
#include <thread>

#include "common/runtime/Database.hpp"
#include "ref_plans.hpp"
#include "runtime_framework.hpp"

typedef Query* (*qnew_t)(QueryConfig*);
typedef void (*qrun_t)(Query*);
typedef void (*qreset_t)(Query*);
typedef void (*qfree_t)(Query*);

int main(int argc, char** argv)
{
	std::string spec, lib, flavor = "hyper", result_file;
	int threads = (int)std::thread::hardware_concurrency();
	int reps = 3;
	bool no_result = false, checksum = false;
	int64_t max_rows = -1;
	size_t vector_size = 1024, morsel_size = 16 * 1024;
	for (int i = 1; i + 1 < argc; i += 2) {
		std::string k = argv[i], v = argv[i + 1];
		if (k == "--workload") spec = v;
		else if (k == "--lib") lib = v;
		else if (k == "--flavor") flavor = v;
		else if (k == "--threads") threads = std::stoi(v);
		else if (k == "--reps") reps = std::stoi(v);
		else if (k == "--result") result_file = v;
		else if (k == "--no-result") no_result = v != "0";
		else if (k == "--checksum") checksum = v != "0";
		else if (k == "--max-rows") max_rows = std::stoll(v);
		else if (k == "--vector-size") vector_size = (size_t)std::stoll(v);
		else if (k == "--morsel-size") morsel_size = (size_t)std::stoll(v);
		else {
			std::cerr << "ref_run: unknown option " << k << std::endl;
			return 2;
		}
	}
	if (spec.empty() || lib.empty() || threads < 1 || reps < 1) {
		std::cerr << "ref_run: --workload and --lib are required" << std::endl;
		return 2;
	}
	try {
		auto w = vc_workload::make(spec);
		runtime::Database db;
		ref_harness::load_workload(db, w, max_rows, threads);

		QueryConfig qconf(db);
		qconf.num_threads = (size_t)threads;
		qconf.vector_size = vector_size;
		qconf.morsel_size = morsel_size;
		qconf.print_result = !no_result;
		/* a CUDA-flavor library ignores the flavor field (the reference has no Flavor::Cuda) */
		qconf.flavor = flavor == "vectorwise" ? QueryConfig::Flavor::Vectorwise : QueryConfig::Flavor::Hyper;

		void* h = dlopen(lib.c_str(), RTLD_NOW);
		if (!h) {
			std::cerr << "ref_run: dlopen failed: " << dlerror() << std::endl;
			return 1;
		}
		auto qnew = (qnew_t)dlsym(h, "voila_query_new");
		auto qrun = (qrun_t)dlsym(h, "voila_query_run");
		auto qreset = (qreset_t)dlsym(h, "voila_query_reset");
		auto qfree = (qfree_t)dlsym(h, "voila_query_free");
		if (!qnew || !qrun || !qreset || !qfree) {
			std::cerr << "ref_run: missing voila_query_* symbols" << std::endl;
			return 1;
		}
		g_config_full_evaluation = qconf.allow_full_evaluation;
		g_config_vector_size = (i64)qconf.vector_size;

		Query* q = qnew(&qconf);
		std::vector<double> times;
		for (int r = 0; r < reps; r++) {
			qreset(q);
			auto t0 = std::chrono::high_resolution_clock::now();
			qrun(q);
			auto t1 = std::chrono::high_resolution_clock::now();
			times.push_back(std::chrono::duration<double, std::milli>(t1 - t0).count());
		}
		if (!result_file.empty()) {
			std::ofstream f(result_file);
			f << q->result.finalize();
		}
		qfree(q);

		std::cout << "{\"times_ms\": [";
		for (size_t i = 0; i < times.size(); i++) {
			std::cout << (i ? ", " : "") << times[i];
		}
		std::cout << "], \"threads\": " << threads << ", \"rows\": " << w.fact_rows;
		if (checksum) {
			std::cout << ", \"checksum\": " << ref_harness::data_checksum(db, w);
		}
		std::cout << "}" << std::endl;
	} catch (const std::exception& e) {
		std::cerr << "ref_run: " << e.what() << std::endl;
		return 1;
	}
	return 0;
}
