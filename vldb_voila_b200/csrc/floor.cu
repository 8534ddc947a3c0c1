/*
 * Streaming-read floor: the fastest plain read of a byte range that this library's kernels
 * are measured against.
 *
 * A pipeline kernel of the CUDA flavor must at least stream its columns from HBM once; the
 * time a bare read of the same byte count takes on the same device, with the same L2 state,
 * is the floor below which no pipeline over those bytes can go.  The kernel below is that
 * bare read: every thread keeps kUnroll independent 16-byte loads in flight (about 64 KiB
 * per SM at full occupancy, well above the bytes-in-flight an HBM3e stack needs to reach its
 * bandwidth), blocks stride over the range in a grid of whole waves, and the words read are
 * folded into one checksum so the loads cannot be removed.
 */
#include <cstdint>
#include <functional>

#include <cuda_runtime.h>

#include "engine_internal.hpp"
#include "../../include/voila_cuda.h"

namespace vc {

int abi_guard_mlp(const std::function<void()>& f);

static constexpr int kFloorThreads = 512;
static constexpr int kUnroll = 8;

__global__ void __launch_bounds__(kFloorThreads) stream_read_kernel(const uint4* __restrict__ src, int64_t n16,
	const unsigned char* __restrict__ tail, int64_t ntail, unsigned long long* out)
{
	uint32_t acc = 0;
	const int64_t stride = (int64_t)gridDim.x * kFloorThreads;
	int64_t i = (int64_t)blockIdx.x * kFloorThreads + threadIdx.x;
	/* kUnroll loads issued before any is consumed */
	for (; i + (kUnroll - 1) * stride < n16; i += kUnroll * stride) {
		uint4 v[kUnroll];
#pragma unroll
		for (int u = 0; u < kUnroll; u++) {
			v[u] = __ldcs(src + i + u * stride);
		}
#pragma unroll
		for (int u = 0; u < kUnroll; u++) {
			acc ^= v[u].x ^ v[u].y ^ v[u].z ^ v[u].w;
		}
	}
	for (; i < n16; i += stride) {
		const uint4 v = __ldcs(src + i);
		acc ^= v.x ^ v.y ^ v.z ^ v.w;
	}
	if (blockIdx.x == 0) {
		for (int64_t t = threadIdx.x; t < ntail; t += kFloorThreads) {
			acc ^= tail[t];
		}
	}
	for (int o = 16; o > 0; o >>= 1) {
		acc ^= __shfl_xor_sync(0xffffffffu, acc, o);
	}
	if ((threadIdx.x & 31u) == 0 && acc) {
		atomicXor(out, (unsigned long long)acc);
	}
}

} // namespace vc

extern "C" int vc_stream_read(const void* device_buf, int64_t bytes, unsigned long long* device_out, void* stream)
{
	return vc::abi_guard_mlp([&] {
		if (!device_buf || !device_out || bytes < 0 || ((uintptr_t)device_buf & 15u)) {
			throw vc::Error(VC_ERR_INVALID, "vc_stream_read needs a 16-byte aligned buffer, an output word and bytes >= 0");
		}
		int dev = 0, sms = 0, occ = 0;
		VC_CHECK_CUDA(cudaGetDevice(&dev));
		VC_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
		VC_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, vc::stream_read_kernel, vc::kFloorThreads, 0));
		const int64_t n16 = bytes / 16;
		const int64_t waves_needed = (n16 + (int64_t)vc::kFloorThreads * vc::kUnroll - 1) / ((int64_t)vc::kFloorThreads * vc::kUnroll);
		int64_t grid = (int64_t)sms * (occ > 0 ? occ : 1);
		if (waves_needed < grid) {
			grid = waves_needed > 0 ? waves_needed : 1;
		}
		vc::stream_read_kernel<<<(unsigned)grid, vc::kFloorThreads, 0, (cudaStream_t)stream>>>(
			(const uint4*)device_buf, n16, (const unsigned char*)device_buf + n16 * 16, bytes - n16 * 16, device_out);
		VC_CHECK_CUDA(cudaGetLastError());
	});
}
