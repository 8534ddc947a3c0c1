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

/* ---------------------------------------------------------------- loads ---------- */

/* Loads rows [r0, r0+V) of a column into registers.  Whole tiles use vector loads through
 * the read-only path (the column base is 16-byte aligned and r0 is a multiple of V);
 * the ragged tail falls back to bounds-checked scalar loads. */
template <typename T, int V>
__device__ __forceinline__ void load_rows(const T* __restrict__ col, int64_t r0, int64_t n, T (&out)[V])
{
	constexpr int bytes = V * (int)sizeof(T);
	if (r0 + V <= n) {
		const T* p = col + r0;
		if constexpr (bytes % 16 == 0) {
			uint4 tmp[bytes / 16];
#pragma unroll
			for (int i = 0; i < bytes / 16; i++) {
				tmp[i] = __ldg(reinterpret_cast<const uint4*>(p) + i);
			}
#pragma unroll
			for (int i = 0; i < V; i++) {
				out[i] = reinterpret_cast<const T*>(tmp)[i];
			}
		} else if constexpr (bytes == 8) {
			uint2 tmp = __ldg(reinterpret_cast<const uint2*>(p));
#pragma unroll
			for (int i = 0; i < V; i++) {
				out[i] = reinterpret_cast<const T*>(&tmp)[i];
			}
		} else if constexpr (bytes == 4) {
			unsigned int tmp = __ldg(reinterpret_cast<const unsigned int*>(p));
#pragma unroll
			for (int i = 0; i < V; i++) {
				out[i] = reinterpret_cast<const T*>(&tmp)[i];
			}
		} else {
#pragma unroll
			for (int i = 0; i < V; i++) {
				out[i] = __ldg(p + i);
			}
		}
	} else {
#pragma unroll
		for (int i = 0; i < V; i++) {
			out[i] = (r0 + i < n) ? __ldg(col + r0 + i) : (T)0;
		}
	}
}

template <typename T>
__device__ __forceinline__ T load_one(const T* __restrict__ col, int64_t row)
{
	return __ldg(col + row);
}

/* ---------------------------------------------------------------- warp helpers --- */

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
	__syncthreads();
	if (lane_id() == 0) {
#pragma unroll
		for (int a = 0; a < A; a++) {
			scratch[warp * A + a] = vals[a];
		}
	}
	__syncthreads();
#pragma unroll
	for (int a = 0; a < A; a++) {
		int64_t s = 0;
		for (unsigned w = 0; w < nw; w++) {
			s += scratch[w * A + a];
		}
		vals[a] = s;
	}
	__syncthreads();
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
		uint4 lo = __ldg(reinterpret_cast<const uint4*>(bk));
		uint4 hi = __ldg(reinterpret_cast<const uint4*>(bk) + 1);
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

template <typename KeyT, typename PayT>
__device__ __forceinline__ bool join_insert(JoinSlot<KeyT, PayT>* __restrict__ slots, uint64_t bucket_mask,
	uint64_t h, KeyT key, PayT pay, unsigned* err)
{
	constexpr int SPB = slots_per_bucket<JoinSlot<KeyT, PayT>>();
	uint64_t b = h & bucket_mask;
	for (int probe = 0; probe < VD_MAX_PROBES; probe++) {
		JoinSlot<KeyT, PayT>* bucket = slots + b * SPB;
#pragma unroll
		for (int s = 0; s < SPB; s++) {
			KeyT* kp = &bucket[s].key;
			if (*(volatile KeyT*)kp == 0) {
				KeyT prev;
				if (sizeof(KeyT) == 4) {
					prev = (KeyT)atomicCAS((unsigned int*)kp, 0u, (unsigned int)key);
				} else {
					prev = (KeyT)atomicCAS((unsigned long long*)kp, 0ull, (unsigned long long)key);
				}
				if (prev == 0) {
					bucket[s].pay = pay;
					return true;
				}
			}
		}
		b = (b + 1) & bucket_mask;
	}
	atomicOr(err, VD_ERR_TABLE_FULL);
	return false;
}

/* ---------------------------------------------------------------- group tables --- */

/*
 * Global group table: `cap` (power of two) slots of (1 + A) 64-bit words: the packed group
 * key + 1 (0 = empty) followed by A aggregate accumulators.  Returns the slot index or -1
 * when the probe sequence is exhausted.
 */
__device__ __forceinline__ int64_t group_find_or_insert(unsigned long long* __restrict__ table, int stride,
	uint64_t mask, uint64_t h, uint64_t stored_key, unsigned* err)
{
	uint64_t i = h & mask;
	for (int probe = 0; probe < VD_MAX_PROBES; probe++) {
		unsigned long long* kp = table + i * (uint64_t)stride;
		unsigned long long cur = *(volatile unsigned long long*)kp;
		if (cur == stored_key) {
			return (int64_t)i;
		}
		if (cur == 0ull) {
			cur = atomicCAS(kp, 0ull, (unsigned long long)stored_key);
			if (cur == 0ull || cur == stored_key) {
				return (int64_t)i;
			}
		}
		i = (i + 1) & mask;
	}
	atomicOr(err, VD_ERR_TABLE_FULL);
	return -1;
}

/* adds the A values of one group (key already packed and +1) into the global group table */
template <int A>
__device__ __forceinline__ void group_add(unsigned long long* __restrict__ table, uint64_t mask, uint64_t h,
	uint64_t stored_key, const int64_t (&vals)[A], unsigned* err)
{
	const int64_t slot = group_find_or_insert(table, 1 + A, mask, h, stored_key, err);
	if (slot >= 0) {
		unsigned long long* row = table + (uint64_t)slot * (1 + A) + 1;
#pragma unroll
		for (int a = 0; a < A; a++) {
			if (vals[a]) {
				atomicAdd(row + a, (unsigned long long)vals[a]);
			}
		}
	}
}

/* Per-CTA shared-memory group cache of S (power of two) slots with the global table's
 * layout.  Returns false when the key finds no slot within 8 probes; the caller then
 * updates the global table directly.  Flushed into the global table at CTA end. */
template <int A>
__device__ __forceinline__ bool cache_add(unsigned long long* cache, int S, uint64_t h, uint64_t stored_key,
	const int64_t (&vals)[A])
{
	uint64_t i = h & (uint64_t)(S - 1);
	for (int probe = 0; probe < 8; probe++) {
		unsigned long long* e = cache + i * (1 + A);
		unsigned long long cur = *(volatile unsigned long long*)e;
		if (cur == 0ull) {
			cur = atomicCAS(e, 0ull, (unsigned long long)stored_key);
			if (cur == 0ull) {
				cur = stored_key;
			}
		}
		if (cur == stored_key) {
#pragma unroll
			for (int a = 0; a < A; a++) {
				if (vals[a]) {
					atomicAdd(e + 1 + a, (unsigned long long)vals[a]);
				}
			}
			return true;
		}
		i = (i + 1) & (uint64_t)(S - 1);
	}
	return false;
}

} // namespace vd

#endif
