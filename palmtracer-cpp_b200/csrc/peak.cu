// FMA-throughput probe used as the denominator of the fit kernels' roofline: every thread runs 8 independent FMA
// chains (no memory traffic), the grid fills every SM several times over, and the rate is timed with CUDA events.
#include <algorithm>

#include "pt_common.cuh"

namespace ptb {

namespace {

template <typename T>
__global__ void __launch_bounds__(256) FmaKernel(T* sink, int iters, T a, T b)
{
	T x0 = static_cast<T>(threadIdx.x), x1 = x0 + T(1), x2 = x0 + T(2), x3 = x0 + T(3);
	T x4 = x0 + T(4), x5 = x0 + T(5), x6 = x0 + T(6), x7 = x0 + T(7);
	for (int i = 0; i < iters; ++i) {
		#pragma unroll
		for (int k = 0; k < 16; ++k) {
			x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
			x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
		}
	}
	const T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
	if (s == T(-1.2345)) { sink[threadIdx.x] = s; }  // keeps the chains alive; never true for these inputs
}

}  // namespace

// Returns FMA-based FLOP/s (2 per FMA) of FP64 (fp64 != 0) or FP32 arithmetic on the current device, or -1.
double MeasureFmaPeak(int fp64)
{
	int dev = 0, sms = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	const int blocks = sms * 8, threads = 256, iters = fp64 ? 256 : 1024;
	void* sink = nullptr;
	if (!PTB_CUDA(cudaMalloc(&sink, 256 * sizeof(double)))) { return -1; }
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	double best = 0;
	for (int rep = 0; rep < 4; ++rep) {
		cudaEventRecord(e0);
		if (fp64) { FmaKernel<double><<<blocks, threads>>>(static_cast<double*>(sink), iters, 0.999999, 1e-7); }
		else { FmaKernel<float><<<blocks, threads>>>(static_cast<float*>(sink), iters, 0.999999f, 1e-7f); }
		cudaEventRecord(e1);
		cudaEventSynchronize(e1);
		float ms = 0;
		cudaEventElapsedTime(&ms, e0, e1);
		const double flops = 2.0 * 8 * 16 * static_cast<double>(iters) * blocks * threads;
		if (rep > 0 && ms > 0) { best = std::max(best, flops / (ms * 1e-3)); }
	}
	CountLaunch(4);
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	cudaFree(sink);
	return PTB_LAUNCHED() ? best : -1;
}

}  // namespace ptb
