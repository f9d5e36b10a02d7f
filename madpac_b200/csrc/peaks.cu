// FMA throughput probe: every thread runs 8 independent dependent-FMA chains in registers; the
// grid fills every SM several times over. Reported in TFLOP/s (an FMA counts 2 flops). It is the
// denominator of the pair kernels' roofline (the pair loop runs on the FP32/FP64 pipes, not on
// tensor cores or HBM).
#include <cuda_runtime.h>

#include "mdgpu.h"

namespace {

template <typename T>
__global__ void __launch_bounds__(256) k_fma_chain(int iters, T a, T b, T* out) {
	T x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
	for (int k = 0; k < iters; k++) {
#pragma unroll
		for (int u = 0; u < 16; u++) {
			x0 = x0 * a + b;
			x1 = x1 * a + b;
			x2 = x2 * a + b;
			x3 = x3 * a + b;
			x4 = x4 * a + b;
			x5 = x5 * a + b;
			x6 = x6 * a + b;
			x7 = x7 * a + b;
		}
	}
	T s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
	if (s == (T) 12345.678) out[0] = s;  // keeps the chains alive
}

template <typename T>
double measure(int sms, T* scratch) {
	const int blocks = sms * 8, threads = 256, iters = 4096;
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	k_fma_chain<T><<<blocks, threads>>>(64, (T) 0.999999, (T) 1e-7, scratch);  // warm-up
	cudaEventRecord(e0);
	k_fma_chain<T><<<blocks, threads>>>(iters, (T) 0.999999, (T) 1e-7, scratch);
	cudaEventRecord(e1);
	cudaEventSynchronize(e1);
	float ms = 0;
	cudaEventElapsedTime(&ms, e0, e1);
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	double flops = 2.0 * 8 * 16 * (double) iters * blocks * threads;
	return flops / (ms * 1e-3) / 1e12;
}

}  // namespace

extern "C" int mdgpu_device_peaks(int device, double* fp32_tflops, double* fp64_tflops) {
	if (cudaSetDevice(device) != cudaSuccess) return MDGPU_ERR_CUDA;
	int sms = 0;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
	void* scratch = nullptr;
	if (cudaMalloc(&scratch, 64) != cudaSuccess) return MDGPU_ERR_CUDA;
	double f32 = measure<float>(sms, (float*) scratch);
	double f64 = measure<double>(sms, (double*) scratch);
	cudaFree(scratch);
	if (cudaGetLastError() != cudaSuccess) return MDGPU_ERR_CUDA;
	if (fp32_tflops) *fp32_tflops = f32;
	if (fp64_tflops) *fp64_tflops = f64;
	return MDGPU_OK;
}
