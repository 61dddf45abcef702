// Fused maximum-likelihood fits for the serving layer: the candidates of several stacks (one chunk each, from the
// server's concurrent slots) are gathered into one device work queue and fitted by ONE persistent fit launch; the
// rows are then scattered back to each chunk's row buffer in its own candidate order. Each candidate's Cand::image
// names its stack, so the fit kernels read its ROI from the right frames. No counterpart in the reference, whose
// frame loop (lib/Palm.cpp:55-70) fits one frame at a time.
#include "engine.h"

namespace ptb {

bool LaunchMle(int lanes, const FitImages& fi, const Cand* cands, const uint32_t* nptr, uint32_t nconst, uint32_t cap,
               const MleParams& mp, double* rows, cudaEvent_t* marks, cudaStream_t st);

namespace {

struct FuseTable {
	int n;
	const Cand* cands[kMaxFitImages];
	const uint32_t* count[kMaxFitImages];  // device candidate counts
	double* rows[kMaxFitImages];
};

// offsets[j] = candidates of the jobs before j (device counts); offsets[n] = the total.
__global__ void FuseOffsets(FuseTable t, uint32_t* offsets)
{
	if (threadIdx.x != 0 || blockIdx.x != 0) { return; }
	uint32_t s = 0;
	for (int j = 0; j < t.n; ++j) {
		offsets[j] = s;
		s += *t.count[j];
	}
	offsets[t.n] = s;
}

__device__ __forceinline__ int JobOf(const uint32_t* offsets, int n, uint32_t k)
{
	int j = 0;
	while (j + 1 < n && k >= offsets[j + 1]) { ++j; }
	return j;
}

__global__ void FuseGather(FuseTable t, const uint32_t* offsets, Cand* fused)
{
	const uint32_t total = offsets[t.n];
	for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
		const int j = JobOf(offsets, t.n, k);
		Cand c = t.cands[j][k - offsets[j]];
		c.image = j;
		fused[k] = c;
	}
}

// One thread per row column: consecutive threads write consecutive doubles of one job's rows.
__global__ void FuseScatter(FuseTable t, const uint32_t* offsets, const double* fusedRows)
{
	const unsigned long long total = static_cast<unsigned long long>(offsets[t.n]) * kCols;
	for (unsigned long long e = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; e < total;
	     e += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
		const uint32_t k = static_cast<uint32_t>(e / kCols);
		const int j = JobOf(offsets, t.n, k);
		t.rows[j][e - static_cast<unsigned long long>(offsets[j]) * kCols] = fusedRows[e];
	}
}

}  // namespace

// Fits the candidates of jobs[0, n) (n <= kMaxFitImages; one fit configuration) in one launch. fusedCands / fusedRows
// hold at least the sum of the jobs' capacities; offsets n + 1 entries; counters 3 unsigned ints (FP64
// re-factorisations and the work-queue counters).
bool LaunchFusedMle(const FitJob* jobs, int n, int lanes, Cand* fusedCands, double* fusedRows, uint32_t* offsets,
                    unsigned int* counters, cudaStream_t st)
{
	if (n < 1 || n > kMaxFitImages) {
		SetError("fused fit: 1 to 16 jobs per launch");
		return false;
	}
	FuseTable t{};
	FitImages fi{};
	t.n = n;
	fi.n = n;
	uint64_t cap = 0;
	for (int j = 0; j < n; ++j) {
		t.cands[j] = jobs[j].cands;
		t.count[j] = jobs[j].count;
		t.rows[j] = jobs[j].rows;
		fi.im[j] = jobs[j].image;
		cap += jobs[j].cap;
	}
	if (cap > 0xffffffffull) {
		SetError("fused fit: more than 2^32 candidates");
		return false;
	}
	MleParams mp = jobs[0].fp.mle;
	mp.fallbacks = counters;
	mp.queue = counters + 1;
	mp.evals = nullptr;
	const int grid = 148 * 4;
	FuseOffsets<<<1, 32, 0, st>>>(t, offsets);
	FuseGather<<<grid, 256, 0, st>>>(t, offsets, fusedCands);
	CountLaunch(2);
	if (!PTB_LAUNCHED()) { return false; }
	if (!LaunchMle(lanes, fi, fusedCands, offsets + n, 0, static_cast<uint32_t>(cap), mp, fusedRows, nullptr, st)) { return false; }
	FuseScatter<<<grid, 256, 0, st>>>(t, offsets, fusedRows);
	CountLaunch();
	return PTB_LAUNCHED();
}

}  // namespace ptb
