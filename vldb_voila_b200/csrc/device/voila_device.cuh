/*
 * Device primitives of the CUDA flavor (sm_100a).
 *
 * Every fused pipeline kernel that the CUDA code generator emits is built from these pieces;
 * the same header is compiled ahead of time by nvcc (generator, MLP and batch kernels) and
 * at query-compile time by NVRTC (pipelines), where it is embedded as a string.
 *
 *   hashing            voila_hash / rehash, bit-identical to runtime.hpp:404-431
 *   column loads       V consecutive rows per thread as 4/8/16-byte vector loads
 *   selection vectors  warp ballot + popc compaction (seltrue, kernel_generator.py:617-631)
 *   warp combining     lanes with equal group keys pre-sum before one lane updates memory
 *   join tables        open addressing in HBM, 32-byte sector buckets, atomicCAS insert
 *   group tables       dense shared-memory slots (small key domains) and an open-addressing
 *                      global table with an optional shared-memory cache (large domains)
 *
 * Error reporting: kernels never trap.  A full table, an exhausted probe sequence or a wait
 * that runs out sets a bit in a device error word that the host reads after the launch.
 */
#ifndef VOILA_B200_DEVICE_CUH
#define VOILA_B200_DEVICE_CUH

#if defined(__CUDACC_RTC__)
typedef unsigned char uint8_t;
typedef signed char int8_t;
typedef short int16_t;
typedef unsigned short uint16_t;
typedef int int32_t;
typedef unsigned int uint32_t;
typedef long long int64_t;
typedef unsigned long long uint64_t;
#else
#include <stdint.h>
#endif

/* error bits written to the device error word */
#define VD_ERR_TABLE_FULL 1u
#define VD_ERR_WAIT_TIMEOUT 2u
#define VD_ERR_BAD_WORK 4u

/* longest probe sequence before a table counts as full */
#define VD_MAX_PROBES 4096

namespace vd {

/* ---------------------------------------------------------------- hashing -------- */

/* voila_hash<T>::hash: three xor-shift-16 steps around two multiplies by 0x45d9f3b,
 * applied to the value widened to u64 (runtime.hpp:413-421). */
__device__ __forceinline__ uint64_t hash(int64_t v)
{
	uint64_t x = (uint64_t)v;
	x ^= x >> 16;
	x *= 0x45d9f3bull;
	x ^= x >> 16;
	x *= 0x45d9f3bull;
	x ^= x >> 16;
	return x;
}

/* voila_hash<T>::rehash: hash(v) ^ (h * 2654435761) (runtime.hpp:423-425) */
__device__ __forceinline__ uint64_t rehash(uint64_t h, int64_t v)
{
	return hash(v) ^ (h * 2654435761ull);
}

/* Table hash of a bit-packed key (flavor hash=mix): the 32-bit finalizer of MurmurHash3
 * (A. Appleby, public domain) for keys of up to 32 bits and the SplitMix64 output function
 * for wider ones.  Both avalanche into the low bits that index the tables and use 32-bit
 * multiplies where they can.  Table positions never reach results, so this cheaper hash
 * may replace voila_hash; both sides of a table use the same one. */
__device__ __forceinline__ uint64_t mix_hash32(uint32_t h)
{
	h ^= h >> 16;
	h *= 0x85ebca6bu;
	h ^= h >> 13;
	h *= 0xc2b2ae35u;
	h ^= h >> 16;
	return (uint64_t)h;
}

__device__ __forceinline__ uint64_t mix_hash64(uint64_t z)
{
	z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
	z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
	return z ^ (z >> 31);
}

/* Gregorian year of a Julian day number (the Calendar FAQ conversion, as runtime.hpp:128-148
 * computes it in unsigned 32-bit steps) */
__device__ __forceinline__ uint32_t julian_year(uint32_t jd)
{
	const uint32_t a = jd + 32044u;
	const uint32_t b = (4u * a + 3u) / 146097u;
	const uint32_t c = a - (146097u * b) / 4u;
	const uint32_t d = (4u * c + 3u) / 1461u;
	const uint32_t e = c - (1461u * d) / 4u;
	const uint32_t m = (5u * e + 2u) / 153u;
	return 100u * b + d - 4800u + m / 10u;
}

/* whether code offset i is in a code set (a bitmap of n bits) */
__device__ __forceinline__ bool code_in(const unsigned* __restrict__ bits, int64_t i, int64_t n)
{
	return (uint64_t)i < (uint64_t)n && ((__ldg(&bits[i >> 5]) >> (unsigned)(i & 31)) & 1u) != 0u;
}

/* product of two values whose ranges fit int32, as one 32x32->64 multiply */
__device__ __forceinline__ int64_t mulw(int64_t a, int64_t b)
{
	return (int64_t)(int32_t)a * (int64_t)(int32_t)b;
}

/* ---------------------------------------------------------------- loads ---------- */

/* A read-only load that does not allocate in L1 (ld.global.nc.L1::no_allocate): column data
 * streamed once leaves L1 to the join and group tables that are probed again. */
template <typename T>
__device__ __forceinline__ T ld_noalloc(const T* p)
{
	if constexpr (sizeof(T) == 16) {
		uint4 r;
		asm("ld.global.nc.L1::no_allocate.v4.u32 {%0, %1, %2, %3}, [%4];"
			: "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w) : "l"(p));
		return *reinterpret_cast<const T*>(&r);
	} else if constexpr (sizeof(T) == 8) {
		unsigned long long r;
		asm("ld.global.nc.L1::no_allocate.u64 %0, [%1];" : "=l"(r) : "l"(p));
		return *reinterpret_cast<const T*>(&r);
	} else if constexpr (sizeof(T) == 4) {
		unsigned r;
		asm("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(r) : "l"(p));
		return *reinterpret_cast<const T*>(&r);
	} else if constexpr (sizeof(T) == 2) {
		unsigned short r;
		asm("ld.global.nc.L1::no_allocate.u16 %0, [%1];" : "=h"(r) : "l"(p));
		return *reinterpret_cast<const T*>(&r);
	} else {
		static_assert(sizeof(T) == 1, "column element of 1, 2, 4, 8 or 16 bytes");
		unsigned short r;
		asm("ld.global.nc.L1::no_allocate.u8 %0, [%1];" : "=h"(r) : "l"(p));
		const unsigned char b = (unsigned char)r;
		return *reinterpret_cast<const T*>(&b);
	}
}

/* One read of column data, by load mode M: 0 through the read-only path from HBM, 1 a
 * coherent L2 load (ld.global.cg) from a column that lives in pinned host memory, 2 the
 * read-only path without L1 allocation (flavor knob stream=noalloc). */
template <int M, typename T>
__device__ __forceinline__ T col_ld(const T* p)
{
	if constexpr (M == 1) {
		return __ldcg(p);
	} else if constexpr (M == 2) {
		return ld_noalloc(p);
	} else {
		return __ldg(p);
	}
}

/* Loads rows [r0, r0+V) of a column into registers.  Whole tiles use vector loads (the
 * column base is 16-byte aligned and r0 is a multiple of V); the ragged tail falls back to
 * bounds-checked scalar loads. */
template <typename T, int V, int M = 0>
__device__ __forceinline__ void load_rows(const T* __restrict__ col, int64_t r0, int64_t n, T (&out)[V])
{
	constexpr int bytes = V * (int)sizeof(T);
	if (r0 + V <= n) {
		const T* p = col + r0;
		if constexpr (bytes % 16 == 0) {
			uint4 tmp[bytes / 16];
#pragma unroll
			for (int i = 0; i < bytes / 16; i++) {
				tmp[i] = col_ld<M>(reinterpret_cast<const uint4*>(p) + i);
			}
#pragma unroll
			for (int i = 0; i < V; i++) {
				out[i] = reinterpret_cast<const T*>(tmp)[i];
			}
		} else if constexpr (bytes == 8) {
			uint2 tmp = col_ld<M>(reinterpret_cast<const uint2*>(p));
#pragma unroll
			for (int i = 0; i < V; i++) {
				out[i] = reinterpret_cast<const T*>(&tmp)[i];
			}
		} else if constexpr (bytes == 4) {
			unsigned int tmp = col_ld<M>(reinterpret_cast<const unsigned int*>(p));
#pragma unroll
			for (int i = 0; i < V; i++) {
				out[i] = reinterpret_cast<const T*>(&tmp)[i];
			}
		} else {
#pragma unroll
			for (int i = 0; i < V; i++) {
				out[i] = col_ld<M>(p + i);
			}
		}
	} else {
#pragma unroll
		for (int i = 0; i < V; i++) {
			out[i] = (r0 + i < n) ? col_ld<M>(col + r0 + i) : (T)0;
		}
	}
}

template <typename T, int M = 0>
__device__ __forceinline__ T load_one(const T* __restrict__ col, int64_t row)
{
	return col_ld<M>(col + row);
}

/* Reads this thread's V consecutive rows of a column tile staged in shared memory. */
template <typename T, int V>
__device__ __forceinline__ void load_rows_smem(const T* s, T (&out)[V])
{
	constexpr int bytes = V * (int)sizeof(T);
	if constexpr (bytes % 16 == 0) {
#pragma unroll
		for (int i = 0; i < bytes / 16; i++) {
			const uint4 tmp = reinterpret_cast<const uint4*>(s)[i];
#pragma unroll
			for (int j = 0; j < 16 / (int)sizeof(T); j++) {
				out[i * (16 / (int)sizeof(T)) + j] = reinterpret_cast<const T*>(&tmp)[j];
			}
		}
	} else if constexpr (bytes == 8) {
		const uint2 tmp = *reinterpret_cast<const uint2*>(s);
#pragma unroll
		for (int i = 0; i < V; i++) {
			out[i] = reinterpret_cast<const T*>(&tmp)[i];
		}
	} else if constexpr (bytes == 4) {
		const unsigned int tmp = *reinterpret_cast<const unsigned int*>(s);
#pragma unroll
		for (int i = 0; i < V; i++) {
			out[i] = reinterpret_cast<const T*>(&tmp)[i];
		}
	} else {
#pragma unroll
		for (int i = 0; i < V; i++) {
			out[i] = s[i];
		}
	}
}

/* ---------------------------------------------------------------- TMA staging ---- */

/*
 * Column tiles are staged into shared memory with bulk asynchronous copies (the untiled
 * cp.async.bulk form of TMA; no cluster multicast) that complete on an mbarrier.  One
 * thread issues copies S-1 tiles ahead of the tile the block is working on, so HBM
 * streaming overlaps the dependent hash-table loads of the current tile.
 */
__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
	return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence()
{
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
		: "memory");
}

/* generic-proxy reads of a stage are ordered before the async-proxy refill of it */
/* One arrival on the barrier (no transaction bytes). */
__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void fence_proxy_async()
{
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

/* global -> shared bulk copy; dst, src 16-byte aligned, bytes a multiple of 16 */
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
		::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
		: "memory");
}

__device__ __forceinline__ uint64_t globaltimer_ns()
{
	uint64_t t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

/* Waits for the barrier's phase with the given parity.  Gives up after `limit_ns` of
 * wall time (returns false) instead of spinning forever. */
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns = 2000000000ull)
{
	const uint32_t a = smem_addr(bar);
	uint64_t start = 0;
	for (uint32_t it = 0;; it++) {
		uint32_t done;
		asm volatile(
			"{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
			: "=r"(done)
			: "r"(a), "r"(parity)
			: "memory");
		if (done) {
			return true;
		}
		if (it == 0) {
			start = globaltimer_ns();
		} else if ((it & 63u) == 0 && globaltimer_ns() - start > limit_ns) {
			return false;
		}
	}
}

/* ---------------------------------------------------------------- warp helpers --- */

/* Block-wide barrier for code whose warps may arrive diverged.  __syncthreads() is the
 * aligned form (bar.sync), which requires every warp to reach it converged; after the
 * per-lane probe loops of the hash tables (early exits, data-dependent trip counts) lanes
 * of a warp can arrive at different times, and on sm_100a an aligned barrier then let
 * warps of one CTA drift onto different work items of the persistent batch kernel.  The
 * non-aligned barrier counts every thread individually. */
__device__ __forceinline__ void block_sync()
{
	asm volatile("barrier.sync 0;" ::: "memory");
}

/* Programmatic dependent launch: pdl_launch_dependents() lets the stream's next kernel be
 * scheduled while this one runs; pdl_wait() blocks until the previous kernel of the stream
 * has completed and its memory is visible.  Both are no-ops for a kernel that was launched
 * without programmatic stream serialization. */
__device__ __forceinline__ void pdl_launch_dependents()
{
	asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ void pdl_wait()
{
	asm volatile("griddepcontrol.wait;" ::: "memory");
}

/* block_sync() that also returns whether any thread passed `v` true (the non-aligned form
 * of __syncthreads_or). */
__device__ __forceinline__ bool block_any(bool v)
{
	unsigned r;
	asm volatile(
		"{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n barrier.red.or.pred q, 0, p;\n selp.u32 %0, 1, 0, q;\n}\n"
		: "=r"(r)
		: "r"((unsigned)v)
		: "memory");
	return r != 0u;
}

__device__ __forceinline__ unsigned lane_id()
{
	return threadIdx.x & 31u;
}

/* Sums the A values of lanes that share `key` into the lowest such lane (the leader).
 * Must be called by all 32 lanes of the warp; lanes with valid == false take part in the
 * shuffles but contribute nothing and never lead. */
template <int A>
__device__ __forceinline__ bool warp_combine(uint64_t key, bool valid, int64_t (&vals)[A])
{
	const unsigned lane = lane_id();
	const uint64_t k = valid ? key : ~0ull;
	const unsigned peers = __match_any_sync(0xffffffffu, k);
	const bool leader = valid && ((peers & ((1u << lane) - 1u)) == 0u);
	unsigned todo = leader ? (peers & ~(1u << lane)) : 0u;
	while (__any_sync(0xffffffffu, todo != 0u)) {
		const int src = todo ? (__ffs(todo) - 1) : (int)lane;
#pragma unroll
		for (int a = 0; a < A; a++) {
			const int64_t x = (int64_t)__shfl_sync(0xffffffffu, (unsigned long long)vals[a], src);
			if (todo) {
				vals[a] += x;
			}
		}
		if (todo) {
			todo &= todo - 1u;
		}
	}
	return leader;
}

/* Bits below the lane: the lanes of a __match_any_sync group whose bit is not set here
 * are the group's lowest lane (its leader). */
__device__ __forceinline__ unsigned lanemask_lt()
{
	return (1u << lane_id()) - 1u;
}

/* Sum of u over the lanes of `mask`, a group found by __match_any_sync (every lane of the
 * group calls with the same mask; the warp's other groups run their own sums in the same
 * instruction).  u has at most BITS significant bits; redux.sync adds 27-bit chunks, which
 * 32 lanes cannot overflow in 32 bits. */
template <int BITS>
__device__ __forceinline__ uint64_t group_sum_u(unsigned mask, uint64_t u)
{
	uint64_t s = __reduce_add_sync(mask, (unsigned)(u & 0x7ffffffu));
	if constexpr (BITS > 27) {
		s += (uint64_t)__reduce_add_sync(mask, (unsigned)((u >> 27) & 0x7ffffffu)) << 27;
	}
	if constexpr (BITS > 54) {
		s += (uint64_t)__reduce_add_sync(mask, (unsigned)(u >> 54)) << 54;
	}
	return s;
}

/* Warp-aggregated append: every lane with `take` gets a distinct position in [0, *cursor),
 * reserved with one atomic per warp. */
__device__ __forceinline__ int64_t warp_append(unsigned long long* cursor, bool take)
{
	const unsigned mask = __ballot_sync(0xffffffffu, take);
	const unsigned lane = lane_id();
	unsigned long long base = 0;
	const int leader = mask ? __ffs(mask) - 1 : 0;
	if (mask && (int)lane == leader) {
		base = atomicAdd(cursor, (unsigned long long)__popc(mask));
	}
	base = __shfl_sync(0xffffffffu, base, leader);
	return (int64_t)base + __popc(mask & ((1u << lane) - 1u));
}

/* Block-aggregated append: one atomic per block and call.  All threads of the block must
 * call it; `scratch` holds at least 33 words of shared memory. */
__device__ __forceinline__ int64_t block_append(unsigned long long* cursor, bool take, unsigned long long* scratch)
{
	const unsigned mask = __ballot_sync(0xffffffffu, take);
	const unsigned lane = lane_id(), warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
	if (lane == 0) {
		scratch[warp] = __popc(mask);
	}
	block_sync();
	if (threadIdx.x == 0) {
		unsigned long long total = 0;
		for (unsigned w = 0; w < nw; w++) {
			const unsigned long long c = scratch[w];
			scratch[w] = total;
			total += c;
		}
		scratch[32] = total ? atomicAdd(cursor, total) : 0ull;
	}
	block_sync();
	const int64_t pos = (int64_t)(scratch[32] + scratch[warp]) + __popc(mask & ((1u << lane) - 1u));
	block_sync();
	return pos;
}

/* Reserves `cnt` consecutive output positions per thread with one atomic per block: returns
 * this thread's first position (threads in order).  All threads call it; `scratch` holds 33
 * words of shared memory. */
__device__ __forceinline__ int64_t block_reserve(unsigned long long* cursor, int cnt, unsigned long long* scratch)
{
	const unsigned lane = lane_id(), warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
	int x = cnt;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const int y = __shfl_up_sync(0xffffffffu, x, o);
		if ((int)lane >= o) {
			x += y;
		}
	}
	if (lane == 31) {
		scratch[warp] = (unsigned long long)x;
	}
	block_sync();
	if (threadIdx.x == 0) {
		unsigned long long run = 0;
		for (unsigned w = 0; w < nw; w++) {
			const unsigned long long c = scratch[w];
			scratch[w] = run;
			run += c;
		}
		scratch[32] = run ? atomicAdd(cursor, run) : 0ull;
	}
	block_sync();
	const int64_t pos = (int64_t)(scratch[32] + scratch[warp]) + x - cnt;
	block_sync();
	return pos;
}

/* Selection vector of the block's active rows (seltrue + compaction, kernel_generator.py
 * :617-631), for survivors collected across tiles: active rows get consecutive positions
 * pos[v] (-1 otherwise) and sel[pos] = their absolute row index r0 + v.  Returns the count.
 * All threads call it; `scan` holds 33 ints of shared memory. */
template <int V, typename R>
__device__ __forceinline__ int block_compact_rows(const bool (&act)[V], int64_t r0, R* sel, int* scan,
	int (&pos)[V])
{
	int cnt = 0;
#pragma unroll
	for (int v = 0; v < V; v++) {
		cnt += act[v] ? 1 : 0;
	}
	const unsigned lane = lane_id(), warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
	int x = cnt;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const int y = __shfl_up_sync(0xffffffffu, x, o);
		if ((int)lane >= o) {
			x += y;
		}
	}
	if (lane == 31) {
		scan[warp] = x;
	}
	block_sync();
	if (threadIdx.x == 0) {
		int run = 0;
		for (unsigned w = 0; w < nw; w++) {
			const int c = scan[w];
			scan[w] = run;
			run += c;
		}
		scan[32] = run;
	}
	block_sync();
	int base = scan[warp] + x - cnt;
#pragma unroll
	for (int v = 0; v < V; v++) {
		if (act[v]) {
			pos[v] = base;
			sel[base] = (R)(r0 + v);
			base++;
		} else {
			pos[v] = -1;
		}
	}
	const int total = scan[32];
	block_sync();
	return total;
}

/* Block dictionary of group slots for per-thread private accumulators: returns the dense
 * code (< gmax) of `slot`, assigning the next code on first sight, or -1 when the block has
 * run out of codes (or another thread's assignment did not become visible within a bounded
 * wait); the caller then falls back to shared-memory atomics, so results never depend on it.
 * dict holds -1 (unseen), -2 (being assigned), -3 (no code) or the code. */
__device__ __forceinline__ int dict_code(int* dict, int* codes, int* ncodes, int64_t slot, int gmax)
{
	int c = *(volatile int*)&dict[slot];
	if (c >= 0) {
		return c;
	}
	if (c == -1) {
		const int old = atomicCAS(&dict[slot], -1, -2);
		if (old == -1) {
			const int k = atomicAdd(ncodes, 1);
			const int code = k < gmax ? k : -3;
			if (k < gmax) {
				codes[k] = (int)slot;
			}
			__threadfence_block();
			atomicExch(&dict[slot], code);
			return code >= 0 ? code : -1;
		}
		c = old;
	}
	for (int spin = 0; c == -2 && spin < 1024; spin++) {
		c = *(volatile int*)&dict[slot];
	}
	return c >= 0 ? c : -1;
}

/* True in every thread of the block that finishes last (all blocks call it once, after
 * their global updates); that block then publishes the final result. */
__device__ __forceinline__ bool last_block_done(unsigned long long* counter, unsigned long long total, int* flag_smem)
{
	__threadfence();
	block_sync();
	if (threadIdx.x == 0) {
		*flag_smem = atomicAdd(counter, 1ull) == total - 1ull;
	}
	block_sync();
	const bool last = *flag_smem != 0;
	if (last) {
		__threadfence();
	}
	return last;
}

/* Block-wide int64 sum (all threads call; result valid in every thread). */
template <int A>
__device__ __forceinline__ void block_sum(int64_t (&vals)[A], int64_t* scratch /* >= 32*A */)
{
#pragma unroll
	for (int a = 0; a < A; a++) {
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) {
			vals[a] += (int64_t)__shfl_xor_sync(0xffffffffu, (unsigned long long)vals[a], o);
		}
	}
	const unsigned warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
	block_sync();
	if (lane_id() == 0) {
#pragma unroll
		for (int a = 0; a < A; a++) {
			scratch[warp * A + a] = vals[a];
		}
	}
	block_sync();
#pragma unroll
	for (int a = 0; a < A; a++) {
		int64_t s = 0;
		for (unsigned w = 0; w < nw; w++) {
			s += scratch[w * A + a];
		}
		vals[a] = s;
	}
	block_sync();
}

/* ---------------------------------------------------------------- join tables ---- */

/*
 * Join hash table: `cap` slots of {key, payload} grouped into 32-byte buckets; KeyT/PayT are
 * uint32_t or uint64_t.  Stored keys are the bit-packed key + 1, so an all-zero table is
 * empty.  Probing starts at bucket (hash & bucket_mask) and walks buckets linearly.
 */
template <typename KeyT, typename PayT>
struct JoinSlot {
	KeyT key;
	PayT pay;
};

template <typename S>
__host__ __device__ __forceinline__ constexpr int slots_per_bucket()
{
	return sizeof(S) >= 32 ? 1 : 32 / (int)sizeof(S);
}

/* buckets for `count` entries: total slots a power of two >= 2 * count (load <= 0.5) */
template <typename S>
__device__ __forceinline__ uint64_t join_buckets(uint64_t count)
{
	const uint64_t spb = (uint64_t)slots_per_bucket<S>();
	uint64_t want = 2 * count;
	if (want < 2 * spb) {
		want = 2 * spb;
	}
	const uint64_t slots = want <= 1 ? 1 : (1ull << (64 - __clzll((long long)(want - 1))));
	return slots / spb;
}

/* One word of a join table: from L2 when the table was built earlier in the same persistent
 * kernel, else through the read-only path. */
template <typename T>
__device__ __forceinline__ T table_ld(const T* p)
{
#ifdef VD_COHERENT_TABLES
	return __ldcg(p);
#else
	return __ldg(p);
#endif
}

/* Dense join tables (packed build key = array index; the key space is small enough that
 * no hashing is needed).  Without payload the table is a bitmap of keys present; with a
 * payload each entry holds payload + 1 (0 = absent) and the first inserted row wins, as in
 * the hash table. */
__device__ __forceinline__ void dense_set(unsigned* bits, uint64_t pk)
{
	atomicOr(&bits[pk >> 5], 1u << (unsigned)(pk & 31u));
}

__device__ __forceinline__ bool dense_test(const unsigned* bits, uint64_t pk)
{
	return ((table_ld(&bits[pk >> 5]) >> (unsigned)(pk & 31u)) & 1u) != 0u;
}

/* Looks `key` up in bucket b: 1 = found (payload in pay), 0 = absent (an empty slot ends the
 * probe sequence), 2 = bucket full without a match (continue with the next bucket). */
template <typename KeyT, typename PayT>
__device__ __forceinline__ int join_probe_bucket(const JoinSlot<KeyT, PayT>* __restrict__ slots, uint64_t b,
	KeyT key, PayT& pay)
{
	typedef JoinSlot<KeyT, PayT> S;
	constexpr int SPB = slots_per_bucket<S>();
	const S* bk = slots + b * SPB;
	S s[SPB];
	if constexpr (sizeof(S) * SPB == 32) {
#ifdef VD_COHERENT_TABLES
		/* the table was built earlier in the same (persistent) kernel: read it from L2 */
		uint4 lo = __ldcg(reinterpret_cast<const uint4*>(bk));
		uint4 hi = __ldcg(reinterpret_cast<const uint4*>(bk) + 1);
#else
		uint4 lo = __ldg(reinterpret_cast<const uint4*>(bk));
		uint4 hi = __ldg(reinterpret_cast<const uint4*>(bk) + 1);
#endif
		reinterpret_cast<uint4*>(s)[0] = lo;
		reinterpret_cast<uint4*>(s)[1] = hi;
	} else {
#pragma unroll
		for (int i = 0; i < SPB; i++) {
			s[i] = bk[i];
		}
	}
#pragma unroll
	for (int i = 0; i < SPB; i++) {
		if (s[i].key == key) {
			pay = s[i].pay;
			return 1;
		}
		if (s[i].key == 0) {
			return 0;
		}
	}
	return 2;
}

/* Inserts into the first free slot of the key's probe sequence.  A table keeps its load at
 * most one half, so a sequence of bucket_mask + 1 buckets always meets a free slot: JoinN
 * tables (duplicate keys cluster) pass that as max_probes, Join01 tables VD_MAX_PROBES. */
template <typename KeyT, typename PayT>
__device__ __forceinline__ bool join_insert(JoinSlot<KeyT, PayT>* __restrict__ slots, uint64_t bucket_mask,
	uint64_t h, KeyT key, PayT pay, unsigned* err, uint64_t max_probes = VD_MAX_PROBES)
{
	constexpr int SPB = slots_per_bucket<JoinSlot<KeyT, PayT>>();
	uint64_t b = h & bucket_mask;
	for (uint64_t probe = 0; probe < max_probes; probe++) {
		JoinSlot<KeyT, PayT>* bucket = slots + b * SPB;
#pragma unroll
		for (int s = 0; s < SPB; s++) {
			/* CAS first: one round trip when the slot is free; a failed CAS observes the
			 * occupant like a read would, and occupied slots stay a prefix of the bucket */
			KeyT* kp = &bucket[s].key;
			KeyT prev;
			if constexpr (sizeof(KeyT) == 4) {
				prev = (KeyT)atomicCAS((unsigned int*)kp, 0u, (unsigned int)key);
			} else {
				prev = (KeyT)atomicCAS((unsigned long long*)kp, 0ull, (unsigned long long)key);
			}
			if (prev == 0) {
				bucket[s].pay = pay;
				return true;
			}
		}
		b = (b + 1) & bucket_mask;
	}
	atomicOr(err, VD_ERR_TABLE_FULL);
	return false;
}

/* ---------------------------------------------------------------- group tables --- */

/*
 * Split group table: the stored keys (packed group key + 1, 0 = empty) in an array of their
 * own, grouped into 32-byte buckets (8 keys of 32 bits or 4 of 64 bits), and the groups'
 * accumulator words in a second array, W 64-bit words per slot.  A probe reads one key sector
 * per bucket; only the group's own slot is touched in the accumulator array.  Several
 * aggregates share one word where their (lower-bound biased, non-negative) sums cannot carry
 * into each other, so one atomic updates them all.
 *
 * Returns the slot of `key` (inserting it into the first free slot of its probe sequence) or
 * -1 when VD_MAX_PROBES buckets hold other keys.  Keys are read from L2 (other CTAs insert
 * concurrently); a slot, once claimed, never changes, and the slots of a bucket fill in
 * order, so a key absent from the occupied prefix of a bucket can only be claimed at or past
 * its first free slot.
 */
template <typename K>
__device__ __forceinline__ int64_t gt_find_or_insert(K* __restrict__ keys, uint64_t bmask, uint64_t h, K key,
	unsigned* err)
{
	constexpr int KPB = 32 / (int)sizeof(K);
	uint64_t b = h & bmask;
	for (int probe = 0; probe < VD_MAX_PROBES; probe++) {
		K* bk = keys + b * KPB;
		K k[KPB];
		const uint4 lo = __ldcg(reinterpret_cast<const uint4*>(bk));
		const uint4 hi = __ldcg(reinterpret_cast<const uint4*>(bk) + 1);
		reinterpret_cast<uint4*>(k)[0] = lo;
		reinterpret_cast<uint4*>(k)[1] = hi;
#pragma unroll
		for (int i = 0; i < KPB; i++) {
			if (k[i] == key) {
				return (int64_t)(b * KPB + i);
			}
		}
#pragma unroll
		for (int i = 0; i < KPB; i++) {
			if (k[i] == 0) {
				K prev;
				if constexpr (sizeof(K) == 4) {
					prev = (K)atomicCAS((unsigned int*)&bk[i], 0u, (unsigned int)key);
				} else {
					prev = (K)atomicCAS((unsigned long long*)&bk[i], 0ull, (unsigned long long)key);
				}
				if (prev == 0 || prev == key) {
					return (int64_t)(b * KPB + i);
				}
			}
		}
		b = (b + 1) & bmask;
	}
	atomicOr(err, VD_ERR_TABLE_FULL);
	return -1;
}

/* gt_find_or_insert whose first bucket (b0, b1: its two 16-byte halves) was loaded ahead */
template <typename K>
__device__ __forceinline__ int64_t gt_find_or_insert_pre(K* __restrict__ keys, uint64_t bmask, uint64_t h, K key,
	uint4 b0, uint4 b1, unsigned* err)
{
	constexpr int KPB = 32 / (int)sizeof(K);
	const uint64_t b = h & bmask;
	K k[KPB];
	reinterpret_cast<uint4*>(k)[0] = b0;
	reinterpret_cast<uint4*>(k)[1] = b1;
	K* bk = keys + b * KPB;
#pragma unroll
	for (int i = 0; i < KPB; i++) {
		if (k[i] == key) {
			return (int64_t)(b * KPB + i);
		}
	}
#pragma unroll
	for (int i = 0; i < KPB; i++) {
		if (k[i] == 0) {
			K prev;
			if constexpr (sizeof(K) == 4) {
				prev = (K)atomicCAS((unsigned int*)&bk[i], 0u, (unsigned int)key);
			} else {
				prev = (K)atomicCAS((unsigned long long*)&bk[i], 0ull, (unsigned long long)key);
			}
			if (prev == 0 || prev == key) {
				return (int64_t)(b * KPB + i);
			}
		}
	}
	/* the bucket is full of other keys: continue from the next one */
	return gt_find_or_insert<K>(keys, bmask, (b + 1) & bmask, key, err);
}

/* adds W packed accumulator words into a slot of the split group table */
template <int W>
__device__ __forceinline__ void gt_add(unsigned long long* __restrict__ acc, int64_t slot, const uint64_t (&w)[W])
{
	unsigned long long* row = acc + (uint64_t)slot * W;
#pragma unroll
	for (int i = 0; i < W; i++) {
		if (w[i]) {
			atomicAdd(row + i, (unsigned long long)w[i]);
		}
	}
}

/* Per-CTA shared-memory cache of S (power of two) slots in the split layout (keys, then
 * S * W words).  Returns false when the key finds no slot within 8 probes; the caller then
 * updates the global table.  Flushed into the global table at the end of the CTA's work. */
template <typename K, int W>
__device__ __forceinline__ bool gt_cache_add(K* ckeys, unsigned long long* cacc, int S, uint64_t h, K key,
	const uint64_t (&w)[W])
{
	uint64_t i = h & (uint64_t)(S - 1);
	for (int probe = 0; probe < 8; probe++) {
		K cur = *(volatile K*)&ckeys[i];
		if (cur == 0) {
			if constexpr (sizeof(K) == 4) {
				cur = (K)atomicCAS((unsigned int*)&ckeys[i], 0u, (unsigned int)key);
			} else {
				cur = (K)atomicCAS((unsigned long long*)&ckeys[i], 0ull, (unsigned long long)key);
			}
			if (cur == 0) {
				cur = key;
			}
		}
		if (cur == key) {
#pragma unroll
			for (int a = 0; a < W; a++) {
				if (w[a]) {
					atomicAdd(cacc + i * W + a, (unsigned long long)w[a]);
				}
			}
			return true;
		}
		i = (i + 1) & (uint64_t)(S - 1);
	}
	return false;
}

/* ------------------------------------------------------------------------------------------
 * Partitioned hash aggregation (flavor aggr=part).
 *
 * Pass 0 runs the pipeline counting each partition's rows per CTA (partition: the high bits
 * of the packed group key's hash) into a CTAs x partitions count matrix; its last CTA turns
 * the totals into partition starts.
 *
 * Pass 1 (the pipeline's main kernel) runs the same grid over the same tiles, so each CTA
 * emits exactly the rows it counted.  It reserves its run in every partition with one atomic
 * on that partition's cursor, then writes each surviving row's record -- the packed group key
 * and each aggregate's value minus its lower bound, bit fields of one or two 64-bit words --
 * at its partition's next position (a shared-memory cursor): every partition's records end
 * up contiguous.
 *
 * Pass 2 (a persistent kernel) takes work items, each one partition or, for a partition
 * holding more than R records, an equal share of its records.  An item aggregates its
 * records into a shared-memory table (keys, then packed accumulator words) and writes the
 * partition's result rows; the items of a split partition leave their groups in a scratch
 * run, and the last of them to finish merges the others' runs before writing the rows.
 * ------------------------------------------------------------------------------------------ */

/* Exclusive prefix sums out[i] = in[0] + ... + in[i-1] over n values held in shared memory
 * (in and out distinct); returns the total.  All threads of the block call it; `scratch`
 * holds 33 words of shared memory. */
__device__ __forceinline__ uint32_t block_excl_scan(const uint32_t* in, uint32_t* out, int n, uint32_t* scratch)
{
	const int T = (int)blockDim.x;
	const int per = (n + T - 1) / T;
	const int b = (int)threadIdx.x * per;
	uint32_t s = 0;
	for (int i = 0; i < per && b + i < n; i++) {
		s += in[b + i];
	}
	const unsigned lane = lane_id(), warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
	uint32_t x = s;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
		if ((int)lane >= o) {
			x += y;
		}
	}
	if (lane == 31) {
		scratch[warp] = x;
	}
	block_sync();
	if (threadIdx.x == 0) {
		uint32_t run = 0;
		for (unsigned w = 0; w < nw; w++) {
			const uint32_t c = scratch[w];
			scratch[w] = run;
			run += c;
		}
		scratch[32] = run;
	}
	block_sync();
	uint32_t pre = scratch[warp] + x - s;
	for (int i = 0; i < per && b + i < n; i++) {
		const uint32_t v = in[b + i];
		out[b + i] = pre;
		pre += v;
	}
	const uint32_t total = scratch[32];
	block_sync();
	return total;
}

/* Exclusive prefix of x over the block's threads, and the block's sum in *total.  All threads
 * call it; `scratch` holds 33 words of shared memory. */
__device__ __forceinline__ uint32_t block_excl_sum(uint32_t x, uint32_t* scratch, uint32_t* total)
{
	const unsigned lane = lane_id(), warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
	uint32_t v = x;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const uint32_t y = __shfl_up_sync(0xffffffffu, v, o);
		if ((int)lane >= o) {
			v += y;
		}
	}
	if (lane == 31) {
		scratch[warp] = v;
	}
	block_sync();
	if (threadIdx.x == 0) {
		uint32_t run = 0;
		for (unsigned w = 0; w < nw; w++) {
			const uint32_t c = scratch[w];
			scratch[w] = run;
			run += c;
		}
		scratch[32] = run;
	}
	block_sync();
	const uint32_t r = scratch[warp] + v - x;
	*total = scratch[32];
	block_sync();
	return r;
}

/* Slot of stored key `key` (packed key + 1) in a shared-memory table of S (power of two)
 * slots, inserting it at the first free slot of its linear probe sequence from h; -1 when
 * every slot holds another key. */
__device__ __forceinline__ int st_find_or_insert(uint32_t* skeys, int S, uint32_t h, uint32_t key)
{
	uint32_t i = h & (uint32_t)(S - 1);
	for (int probe = 0; probe < S; probe++) {
		uint32_t cur = *(volatile uint32_t*)&skeys[i];
		if (cur == 0u) {
			cur = atomicCAS(&skeys[i], 0u, key);
			if (cur == 0u) {
				return (int)i;
			}
		}
		if (cur == key) {
			return (int)i;
		}
		i = (i + 1) & (uint32_t)(S - 1);
	}
	return -1;
}

/* the largest p < n with pre[p] <= x (pre non-decreasing, pre[0] = 0 <= x) */
__device__ __forceinline__ int last_at_most(const uint32_t* pre, int n, uint32_t x)
{
	int lo = 0, hi = n - 1;
	while (lo < hi) {
		const int mid = (lo + hi + 1) >> 1;
		if (pre[mid] <= x) {
			lo = mid;
		} else {
			hi = mid - 1;
		}
	}
	return lo;
}

} // namespace vd

#endif
