/*
 * Minimal stand-in for the parts of Intel TBB that the reference's runtime uses on the
 * query path (test infrastructure only: TBB is not installed in this image).
 *
 * Used by: runtime_framework.cpp:192 (tbb::parallel_for over num_threads),
 * main.cpp:118 / explorer.cpp:680 (tbb::task_scheduler_init) and
 * db-engine-paradigms/include/common/runtime/Concurrency.hpp:80 (tbb::task_group).
 *
 * parallel_for runs one std::thread per index so that the reference's num_threads
 * workers really run concurrently, as TBB would schedule them.
 */
#ifndef VOILA_ORACLE_TBB_SHIM_H
#define VOILA_ORACLE_TBB_SHIM_H

#include <cstddef>
#include <functional>
#include <thread>
#include <vector>

namespace tbb {

struct task_scheduler_init {
	static const int automatic = -1;
	explicit task_scheduler_init(int = automatic) {}
	static int default_num_threads() { return (int)std::thread::hardware_concurrency(); }
};

template <typename Index, typename Func>
void parallel_for(Index first, Index last, Index step, const Func& f)
{
	std::vector<std::thread> workers;
	for (Index i = first; i < last; i += step) {
		workers.emplace_back([&f, i]() { f(i); });
	}
	for (auto& w : workers) {
		w.join();
	}
}

template <typename Index, typename Func>
void parallel_for(Index first, Index last, const Func& f)
{
	parallel_for<Index, Func>(first, last, (Index)1, f);
}

class task_group {
	std::vector<std::thread> workers;
public:
	template <typename F> void run(const F& f) { workers.emplace_back(f); }
	void wait() {
		for (auto& w : workers) {
			if (w.joinable()) w.join();
		}
		workers.clear();
	}
	~task_group() { wait(); }
};

} // namespace tbb

#endif
