/*
 * Seeded, counter-based synthetic column generator.
 *
 * Every value is a pure function of (column seed, row index), so the same bytes come out of
 * the host (C/C++: the product's upload path, the oracle and the reference harness) and the
 * device (the generator kernel used for the large resident workloads), in any order and in
 * parallel.  Stands in for the TPC-H/SSB loaders of the reference
 * (db-engine-paradigms/src/common/runtime/Import.cpp:165-250), whose data is not available.
 *
 * Random bits: the SplitMix64 output function (Steele, Lea, Flood 2014; public-domain
 * reference by S. Vigna) applied to a Weyl sequence seeded per column.
 */
#ifndef VOILA_B200_DATAGEN_H
#define VOILA_B200_DATAGEN_H

#include <stdint.h>

#if defined(__CUDACC__) || defined(__CUDACC_RTC__)
#define VC_GEN_FN __host__ __device__ __forceinline__
#else
#define VC_GEN_FN static inline
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* column types shared by the C ABI, the generator and the codegen */
enum {
	VC_TYPE_U8 = 1,
	VC_TYPE_I16 = 2,
	VC_TYPE_I32 = 3,
	VC_TYPE_I64 = 4,
	VC_TYPE_STR = 5 /* variable-length string; on the device a 32-bit dictionary code */
};

/* longest generated string (host output rows are VC_GEN_STR_WIDTH bytes, NUL-padded) */
#define VC_GEN_STR_WIDTH 32

/* generator kinds */
enum {
	VC_GEN_UNIFORM = 0, /* uniform integer in [a, b] */
	VC_GEN_SEQ = 1,     /* a + row */
	VC_GEN_PERM = 2,    /* a + perm(row), perm a seeded bijection of [0, n) */
	VC_GEN_ZIPF = 3,    /* key in [1, b] with P(k) ~ k^-s; s == 0 means uniform */
	VC_GEN_CHOICE = 4,  /* one of b byte values packed little-endian into a (b <= 8) */
	VC_GEN_DIV = 5,     /* a + (row * c) / b */
	VC_GEN_MOD = 6,     /* a + row % b */
	VC_GEN_WORDS = 7    /* a words (1..4) drawn from the first b (1..24) of a word list, space-separated */
};

typedef struct vc_gen_spec {
	int32_t kind;
	int32_t type;
	int64_t a;
	int64_t b;
	int64_t c;
	double s;
	uint64_t seed;
	int64_t n; /* table cardinality (PERM domain) */
} vc_gen_spec;

VC_GEN_FN uint64_t vc_gen_mix64(uint64_t z)
{
	z = (z ^ (z >> 30)) * UINT64_C(0xbf58476d1ce4e5b9);
	z = (z ^ (z >> 27)) * UINT64_C(0x94d049bb133111eb);
	return z ^ (z >> 31);
}

/* i-th output of the column's Weyl-sequence generator */
VC_GEN_FN uint64_t vc_gen_bits(uint64_t seed, uint64_t i)
{
	const uint64_t base = vc_gen_mix64(seed ^ UINT64_C(0x6a09e667f3bcc909));
	return vc_gen_mix64(base + (i + 1) * UINT64_C(0x9e3779b97f4a7c15));
}

/* uniform in [0, range): for range <= 2^32 from the top 32 bits (multiply-shift); wider
 * ranges take the high half of the full 64 x 64-bit product */
VC_GEN_FN uint64_t vc_gen_below(uint64_t bits, uint64_t range)
{
	if (range <= (UINT64_C(1) << 32)) {
		return ((bits >> 32) * range) >> 32;
	}
	return (uint64_t)(((unsigned __int128)bits * range) >> 64);
}

/* 4-round balanced Feistel bijection on [0, 4^h), cycle-walked into [0, n) */
VC_GEN_FN uint64_t vc_gen_perm(uint64_t seed, uint64_t n, uint64_t x)
{
	int h = 1;
	while ((UINT64_C(1) << (2 * h)) < n) {
		h++;
	}
	const uint64_t mask = (UINT64_C(1) << h) - 1;
	do {
		uint64_t l = x >> h, r = x & mask;
		for (uint64_t round = 0; round < 4; round++) {
			const uint64_t f = vc_gen_mix64(seed + round * UINT64_C(0x9e3779b97f4a7c15) + r) & mask;
			const uint64_t nl = r;
			r = l ^ f;
			l = nl;
		}
		x = (l << h) | r;
	} while (x >= n);
	return x;
}

/* number of cdf entries <= u, i.e. the 0-based rank whose bucket holds u */
VC_GEN_FN int64_t vc_gen_zipf_rank(const double* cdf, int64_t n, double u)
{
	int64_t lo = 0, hi = n;
	while (lo < hi) {
		const int64_t mid = lo + ((hi - lo) >> 1);
		if (cdf[mid] <= u) {
			lo = mid + 1;
		} else {
			hi = mid;
		}
	}
	return lo < n ? lo : n - 1;
}

/* value of row `row` as int64 (before narrowing to spec->type) */
VC_GEN_FN int64_t vc_gen_value(const vc_gen_spec* spec, const double* zipf_cdf, int64_t row)
{
	const uint64_t bits = vc_gen_bits(spec->seed, (uint64_t)row);
	switch (spec->kind) {
	case VC_GEN_UNIFORM:
		return spec->a + (int64_t)vc_gen_below(bits, (uint64_t)(spec->b - spec->a + 1));
	case VC_GEN_SEQ:
		return spec->a + row;
	case VC_GEN_PERM:
		return spec->a + (int64_t)vc_gen_perm(spec->seed, (uint64_t)spec->n, (uint64_t)row);
	case VC_GEN_ZIPF:
		if (spec->s == 0.0 || !zipf_cdf) {
			return 1 + (int64_t)vc_gen_below(bits, (uint64_t)spec->b);
		} else {
			const double u = (double)(bits >> 11) * (1.0 / 9007199254740992.0);
			return 1 + vc_gen_zipf_rank(zipf_cdf, spec->b, u);
		}
	case VC_GEN_CHOICE: {
		const uint64_t k = vc_gen_below(bits, (uint64_t)spec->b);
		return (int64_t)(((uint64_t)spec->a >> (8 * k)) & 0xff);
	}
	case VC_GEN_DIV:
		return spec->a + (row * spec->c) / spec->b;
	case VC_GEN_MOD:
		return spec->a + row % spec->b;
	default:
		return 0;
	}
}

VC_GEN_FN int vc_gen_type_size(int32_t type)
{
	return type == VC_TYPE_U8 ? 1 : type == VC_TYPE_I16 ? 2 : (type == VC_TYPE_I32 || type == VC_TYPE_STR) ? 4 : 8;
}

VC_GEN_FN void vc_gen_store(int32_t type, void* out, int64_t i, int64_t v)
{
	switch (type) {
	case VC_TYPE_U8: ((uint8_t*)out)[i] = (uint8_t)v; break;
	case VC_TYPE_I16: ((int16_t*)out)[i] = (int16_t)v; break;
	case VC_TYPE_I32: ((int32_t*)out)[i] = (int32_t)v; break;
	default: ((int64_t*)out)[i] = v; break;
	}
}

#if !defined(__CUDACC_RTC__) && !defined(__CUDA_ARCH__)
#include <math.h>
#include <string.h>

/* String of row `row` of a VC_GEN_WORDS column, NUL-terminated, at most VC_GEN_STR_WIDTH - 1
 * characters; returns its length.  Host only: strings are dictionary-encoded when uploaded. */
static inline int vc_gen_string(const vc_gen_spec* spec, int64_t row, char* out)
{
	static const char* const words[24] = {"amber", "azure", "beige", "black", "blue", "coral", "cream", "cyan",
		"gold", "green", "grey", "indigo", "ivory", "khaki", "lime", "navy", "olive", "orange", "pink", "plum",
		"red", "rose", "tan", "white"};
	const uint64_t bits = vc_gen_bits(spec->seed, (uint64_t)row);
	const int64_t nwords = spec->a < 1 ? 1 : (spec->a > 4 ? 4 : spec->a);
	const uint64_t choices = (uint64_t)(spec->b < 1 ? 1 : (spec->b > 24 ? 24 : spec->b));
	int len = 0;
	for (int64_t j = 0; j < nwords; j++) {
		const char* w = words[((bits >> (16 * j)) & 0xffff) % choices];
		const int wl = (int)strlen(w);
		if (j) {
			out[len++] = ' ';
		}
		memcpy(out + len, w, (size_t)wl);
		len += wl;
	}
	out[len] = 0;
	return len;
}
/*
 * Inverse-CDF table for VC_GEN_ZIPF: cdf[k-1] = sum_{j<=k} j^-s / sum_{j<=n} j^-s.
 * Host only; the device generator receives the finished table.  Built with one left-to-right
 * summation and no fused multiply-add, so every build of this header yields the same doubles.
 */
static inline void vc_gen_build_zipf_cdf(double s, int64_t n, double* cdf)
{
	double acc = 0.0;
	for (int64_t k = 1; k <= n; k++) {
		acc = acc + pow((double)k, -s);
		cdf[k - 1] = acc;
	}
	for (int64_t k = 0; k < n; k++) {
		cdf[k] = cdf[k] / acc;
	}
	cdf[n - 1] = 1.0;
}
#endif

#ifdef __cplusplus
}
#endif

#endif
