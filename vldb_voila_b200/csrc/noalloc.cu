/*
 * Allocation-free variant of the hash join + global aggregate pipeline.
 *
 * vc_join_aggr_noalloc runs the same computation as a join_aggr query (filter the build side
 * on attr < threshold, Join01 probe on the key, sum(val) and count over the matches) for
 * callers that cannot allocate device memory: code running where cudaMalloc is forbidden or
 * unsafe, such as inside a host callback or under an allocator that owns all device memory,
 * or callers that must not add allocations of their own.  The caller passes the inputs and
 * the output; the join table and the accumulators -- the only scratch memory the pipeline
 * needs -- live in file-scope device arrays below, so the call performs no cudaMalloc,
 * cudaFree or other allocating call.
 *
 * Limits and sharing: the table has kNoAllocSlots slots, so at most kNoAllocSlots / 2 build
 * rows are accepted (larger inputs are rejected with VC_ERR_INVALID before any work).  Every
 * GPU that loads the library holds these arrays (32 MiB + 64 B) until the process exits.
 * All calls on a device share them and the last call's contents remain: each call clears the
 * part it uses, and calls that overlap on the GPU (different streams, or graphs replayed
 * concurrently) race on the shared table and give wrong results.
 */
#include <algorithm>
#include <cstdint>
#include <functional>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "engine_internal.hpp"
#include "../../include/voila_cuda.h"

namespace vc {

int abi_guard_mlp(const std::function<void()>& f);

static constexpr int64_t kNoAllocSlots = int64_t(1) << 22; /* 4 Mi slots of 8 bytes: 32 MiB */

/* join table: slot = (1 << 32) | (uint32)key, 0 = empty */
static __device__ __align__(256) unsigned long long g_noalloc_table[kNoAllocSlots];
/* [0] sum, [1] count, [2] error bits */
static __device__ __align__(256) unsigned long long g_noalloc_acc[8];

__device__ __forceinline__ uint64_t noalloc_hash(uint32_t k)
{
	/* MurmurHash3 32-bit finalizer (A. Appleby, public domain) */
	k ^= k >> 16;
	k *= 0x85ebca6bu;
	k ^= k >> 13;
	k *= 0xc2b2ae35u;
	k ^= k >> 16;
	return k;
}

__global__ void __launch_bounds__(256) noalloc_clear(unsigned long long* table, int64_t slots, unsigned long long* acc)
{
	const int64_t stride = (int64_t)gridDim.x * blockDim.x;
	for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < slots; i += stride) {
		table[i] = 0ull;
	}
	if (blockIdx.x == 0 && threadIdx.x < 8) {
		acc[threadIdx.x] = 0ull;
	}
}

__global__ void __launch_bounds__(256) noalloc_build(const int32_t* __restrict__ key, const int32_t* __restrict__ attr,
	int64_t n, int32_t thr, unsigned long long* table, uint64_t mask, unsigned long long* acc)
{
	const int64_t stride = (int64_t)gridDim.x * blockDim.x;
	for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
		if (attr[i] >= thr) {
			continue;
		}
		const unsigned long long stored = (1ull << 32) | (uint32_t)key[i];
		uint64_t s = noalloc_hash((uint32_t)key[i]) & mask;
		int probe = 0;
		for (; probe <= (int)mask && probe < 1 << 20; probe++) {
			const unsigned long long prev = atomicCAS(&table[s], 0ull, stored);
			if (prev == 0ull || prev == stored) {
				break; /* inserted, or a duplicate key (Join01 keeps one) */
			}
			s = (s + 1) & mask;
		}
		if (probe > (int)mask || probe >= 1 << 20) {
			atomicOr(&acc[2], 1ull);
		}
	}
}

__global__ void __launch_bounds__(256) noalloc_probe(const int32_t* __restrict__ key, const int64_t* __restrict__ val,
	int64_t n, const unsigned long long* __restrict__ table, uint64_t mask, unsigned long long* acc)
{
	unsigned long long sum = 0, cnt = 0;
	const int64_t stride = (int64_t)gridDim.x * blockDim.x;
	for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
		const unsigned long long want = (1ull << 32) | (uint32_t)key[i];
		uint64_t s = noalloc_hash((uint32_t)key[i]) & mask;
		for (int probe = 0; probe <= (int)mask && probe < 1 << 20; probe++) {
			const unsigned long long cur = __ldg(&table[s]);
			if (cur == want) {
				sum += (unsigned long long)val[i];
				cnt += 1;
				break;
			}
			if (cur == 0ull) {
				break;
			}
			s = (s + 1) & mask;
		}
	}
	for (int o = 16; o > 0; o >>= 1) {
		sum += __shfl_xor_sync(0xffffffffu, sum, o);
		cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
	}
	if ((threadIdx.x & 31) == 0 && cnt) {
		atomicAdd(&acc[0], sum);
		atomicAdd(&acc[1], cnt);
	}
}

__global__ void noalloc_finish(const unsigned long long* acc, int64_t* out)
{
	if (threadIdx.x == 0) {
		out[0] = (int64_t)acc[0];
		out[1] = (int64_t)acc[1];
		out[2] = (int64_t)acc[2];
	}
}

/* Device addresses of the static arrays, looked up once per device (cudaGetSymbolAddress
 * with that device current).  The host-side names of the arrays are not device addresses. */
struct NoAllocAddrs {
	unsigned long long* table = nullptr;
	unsigned long long* acc = nullptr;
};

static NoAllocAddrs noalloc_addrs(int device)
{
	static std::mutex mu;
	static NoAllocAddrs cache[128];
	if (device < 0 || device >= 128) {
		throw Error(VC_ERR_INVALID, "device index out of range");
	}
	std::lock_guard<std::mutex> g(mu);
	NoAllocAddrs& a = cache[device];
	if (!a.table) {
		void* t = nullptr;
		void* c = nullptr;
		VC_CHECK_CUDA(cudaGetSymbolAddress(&t, g_noalloc_table));
		VC_CHECK_CUDA(cudaGetSymbolAddress(&c, g_noalloc_acc));
		a.table = (unsigned long long*)t;
		a.acc = (unsigned long long*)c;
	}
	return a;
}

} // namespace vc

extern "C" int vc_join_aggr_noalloc(const int32_t* build_key, const int32_t* build_attr, int64_t build_rows,
	int32_t attr_threshold, const int32_t* probe_key, const int64_t* probe_val, int64_t probe_rows, int64_t* out,
	void* stream)
{
	return vc::abi_guard_mlp([&] {
		using namespace vc;
		if (build_rows < 0 || probe_rows < 0 || !out || (build_rows && (!build_key || !build_attr)) ||
			(probe_rows && (!probe_key || !probe_val))) {
			throw Error(VC_ERR_INVALID, "bad arguments");
		}
		if (build_rows > kNoAllocSlots / 2) {
			throw Error(VC_ERR_INVALID, "vc_join_aggr_noalloc takes at most " + std::to_string(kNoAllocSlots / 2) +
				" build rows (its static join table has " + std::to_string(kNoAllocSlots) + " slots)");
		}
		int dev = 0;
		VC_CHECK_CUDA(cudaGetDevice(&dev));
		const NoAllocAddrs a = noalloc_addrs(dev);
		int64_t slots = 64;
		while (slots < 2 * build_rows) {
			slots <<= 1;
		}
		const uint64_t mask = (uint64_t)slots - 1;
		int sms = 0;
		VC_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
		cudaStream_t s = (cudaStream_t)stream;
		auto grid = [&](int64_t n) {
			int64_t g = (n + 255) / 256;
			return (unsigned)std::max<int64_t>(1, std::min<int64_t>(g, (int64_t)sms * 8));
		};
		noalloc_clear<<<grid(slots), 256, 0, s>>>(a.table, slots, a.acc);
		if (build_rows) {
			noalloc_build<<<grid(build_rows), 256, 0, s>>>(build_key, build_attr, build_rows, attr_threshold, a.table,
				mask, a.acc);
		}
		if (probe_rows) {
			noalloc_probe<<<grid(probe_rows), 256, 0, s>>>(probe_key, probe_val, probe_rows, a.table, mask, a.acc);
		}
		noalloc_finish<<<1, 32, 0, s>>>(a.acc, out);
		VC_CHECK_CUDA(cudaGetLastError());
	});
}
