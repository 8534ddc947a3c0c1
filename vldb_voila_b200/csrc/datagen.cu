/*
 * Ahead-of-time generator kernel: fills a column on the device with the same values the
 * host generator (datagen.h) produces, so resident workloads of billions of rows need no
 * host->device copy.  Grid-stride, one value per thread step.
 */
#include <cuda_runtime.h>

#include "datagen.h"

namespace vc {

template <typename T>
__global__ void __launch_bounds__(256) generate_kernel(T* __restrict__ out, vc_gen_spec spec,
	const double* __restrict__ cdf, int64_t rows)
{
	for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += (int64_t)gridDim.x * blockDim.x) {
		out[i] = (T)vc_gen_value(&spec, cdf, i);
	}
}

cudaError_t launch_generate(void* out, const vc_gen_spec& spec, const double* zipf_cdf_dev, int64_t rows,
	cudaStream_t stream)
{
	if (rows <= 0) {
		return cudaSuccess;
	}
	int dev = 0, sms = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	int64_t blocks = (rows + 255) / 256;
	if (blocks > (int64_t)sms * 16) {
		blocks = (int64_t)sms * 16;
	}
	switch (spec.type) {
	case VC_TYPE_U8:
		generate_kernel<uint8_t><<<(unsigned)blocks, 256, 0, stream>>>((uint8_t*)out, spec, zipf_cdf_dev, rows);
		break;
	case VC_TYPE_I16:
		generate_kernel<int16_t><<<(unsigned)blocks, 256, 0, stream>>>((int16_t*)out, spec, zipf_cdf_dev, rows);
		break;
	case VC_TYPE_I32:
		generate_kernel<int32_t><<<(unsigned)blocks, 256, 0, stream>>>((int32_t*)out, spec, zipf_cdf_dev, rows);
		break;
	default:
		generate_kernel<int64_t><<<(unsigned)blocks, 256, 0, stream>>>((int64_t*)out, spec, zipf_cdf_dev, rows);
		break;
	}
	return cudaGetLastError();
}

} // namespace vc
