// Candidate construction from region sums, per-frame (Y, X) ordering of fitted rows and final row numbering.
//
// Reference: SegmentationInfo fields from ComputeStatistics (Segmentation2D.cpp:144-175); per-frame sort with
// std::weak_order on Y then X (FrameProcessor.cpp:35-39); Id / Plane / Index assignment (lib/Palm.cpp:24-43).
#include "pt_common.cuh"

namespace ptb {

namespace {

// Region sums are exact integers in 2^-16 units, so x = sum(v j) / sum(v) is the reference's FP64 quotient exactly.
__global__ void BuildCandidates(Workspace ws)
{
	const uint32_t n = min(ws.cnt->nfit, ws.capRows);
	for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
		const uint32_t r = ws.candRegion[k];
		const double sv = static_cast<double>(ws.regSumV[r]);
		Cand c;
		c.x = static_cast<double>(ws.regSumVJ[r]) / sv;
		c.y = static_cast<double>(ws.regSumVI[r]) / sv;
		c.intensity = sv * kW1Unit;
		c.surf = static_cast<double>(ws.regCount[r]);
		c.frame = static_cast<int>(ws.candFrame[k]);
		c.image = 0;
		ws.cand[k] = c;
	}
}

// Total order of std::weak_order on doubles: -NaN < -inf < ... < -0 == +0 < ... < +inf < +NaN.
__device__ __forceinline__ unsigned long long WeakKey(double d)
{
	if (d == 0.0) { d = 0.0; }
	unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(d));
	if (isnan(d)) { return (b >> 63) ? 0ull : ~0ull; }
	return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

constexpr int kSortThreads = 512;
constexpr int kSmemSort = 4096;  // rows sorted in shared memory (80 KB); larger frames sort in global scratch
constexpr size_t kSortSmemBytes = kSmemSort * (2 * sizeof(unsigned long long) + sizeof(uint32_t));

__device__ __forceinline__ bool KeyLess(unsigned long long ya, unsigned long long xa, unsigned long long yb, unsigned long long xb)
{
	return ya < yb || (ya == yb && xa < xb);
}

// Bitonic sort of (ky, kx, idx) over a power-of-two length `len`; entries >= n hold +inf keys.
template <bool SMEM>
__device__ void Bitonic(unsigned long long* ky, unsigned long long* kx, uint32_t* id, uint32_t len)
{
	for (uint32_t size = 2; size <= len; size <<= 1) {
		for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
			for (uint32_t t = threadIdx.x; t < len / 2; t += blockDim.x) {
				const uint32_t lo = 2 * t - (t & (stride - 1));
				const uint32_t hi = lo + stride;
				const bool up = (lo & size) == 0;
				const bool swap = up ? KeyLess(ky[hi], kx[hi], ky[lo], kx[lo]) : KeyLess(ky[lo], kx[lo], ky[hi], kx[hi]);
				if (swap) {
					const unsigned long long a = ky[lo], b = kx[lo];
					const uint32_t c = id[lo];
					ky[lo] = ky[hi]; kx[lo] = kx[hi]; id[lo] = id[hi];
					ky[hi] = a; kx[hi] = b; id[hi] = c;
				}
			}
			if (SMEM) { __syncthreads(); }
			else { __syncthreads(); __threadfence_block(); }
		}
	}
}

// One CTA per frame: sort that frame's rows by (Y, X) and write them numbered to out (device memory). Ids continue
// from *rowBase (rows written by earlier chunks); with offsetOut the rows also land at out + *rowBase rows.
__global__ void __launch_bounds__(kSortThreads) SortFrames(Workspace ws, double* out, const unsigned long long* rowBase,
                                                            int offsetOut, unsigned long long planeBase, uint32_t capScratch)
{
	extern __shared__ __align__(16) unsigned long long sortSmem[];
	unsigned long long* sy = sortSmem;
	unsigned long long* sx = sy + kSmemSort;
	uint32_t* si = reinterpret_cast<uint32_t*>(sx + kSmemSort);
	const int f = blockIdx.x;
	const uint32_t base = ws.frameOutBase[f];
	const uint32_t n = ws.frameOutBase[f + 1] - base;
	if (n == 0) { return; }
	uint32_t len = 1;
	while (len < n) { len <<= 1; }
	const double* __restrict__ rows = ws.rows + static_cast<long long>(base) * kCols;
	unsigned long long *ky, *kx;
	uint32_t* id;
	const bool smem = len <= static_cast<uint32_t>(kSmemSort);
	if (smem) { ky = sy; kx = sx; id = si; }
	else {
		// global scratch of this frame: 2 * len keys from 4 * base and len indices from 2 * base (len < 2 n, so frames
		// never overlap; the key scratch holds 4 * capRows and the index scratch 2 * capRows entries)
		if (4ull * base + 2ull * len > 4ull * capScratch) { return; }
		ky = reinterpret_cast<unsigned long long*>(ws.sortKey) + 4ull * base;
		kx = ky + len;
		id = ws.sortIdx + 2ull * base;
	}
	// keys: four rows per thread and pass, their loads issued before any key is stored
	for (uint32_t i0 = threadIdx.x; i0 < len; i0 += 4 * blockDim.x) {
		double y[4], x[4];
		#pragma unroll
		for (int u = 0; u < 4; ++u) {
			const uint32_t i = i0 + u * blockDim.x;
			y[u] = x[u] = 0.0;
			if (i < n) {
				y[u] = __ldg(rows + static_cast<long long>(i) * kCols + cY);
				x[u] = __ldg(rows + static_cast<long long>(i) * kCols + cX);
			}
		}
		#pragma unroll
		for (int u = 0; u < 4; ++u) {
			const uint32_t i = i0 + u * blockDim.x;
			if (i < len) {
				ky[i] = i < n ? WeakKey(y[u]) : ~0ull;
				kx[i] = i < n ? WeakKey(x[u]) : ~0ull;
				id[i] = i;
			}
		}
	}
	__syncthreads();
	if (smem) { Bitonic<true>(ky, kx, id, len); }
	else { Bitonic<false>(ky, kx, id, len); }
	const unsigned long long idBase = *rowBase;
	double* __restrict__ dst = out + (offsetOut ? static_cast<long long>(idBase) * kCols : 0ll) + static_cast<long long>(base) * kCols;
	// numbered rows in sorted order, element by element (consecutive threads: consecutive columns of a row, then the
	// next row), four elements per thread and pass with their loads issued first
	const double plane = static_cast<double>(planeBase + f + 1);
	const uint32_t total = n * static_cast<uint32_t>(kCols);
	for (uint32_t e0 = threadIdx.x; e0 < total; e0 += 4 * blockDim.x) {
		double v[4];
		#pragma unroll
		for (int u = 0; u < 4; ++u) {
			const uint32_t e = e0 + u * blockDim.x;
			v[u] = 0.0;
			if (e < total) {
				const uint32_t i = e / kCols, c = e - i * kCols;
				v[u] = __ldg(rows + static_cast<long long>(id[i]) * kCols + c);
			}
		}
		#pragma unroll
		for (int u = 0; u < 4; ++u) {
			const uint32_t e = e0 + u * blockDim.x;
			if (e < total) {
				const uint32_t i = e / kCols, c = e - i * kCols;
				dst[e] = c == cId ? static_cast<double>(idBase + base + i + 1) : c == cPlane ? plane : c == cIndex ? static_cast<double>(i + 1) : v[u];
			}
		}
	}
}

// After SortFrames: the chunk's rows join the running count.
__global__ void AdvanceRowBase(Workspace ws, unsigned long long* rowBase)
{
	*rowBase += ws.frameOutBase[ws.g.B];
}

}  // namespace

bool LaunchBuildCandidates(const Workspace& ws, cudaStream_t st)
{
	BuildCandidates<<<148 * 4, 256, 0, st>>>(ws);
	CountLaunch();
	return PTB_LAUNCHED();
}

// out: device destination of the rows. rowBase: device count of the rows written by earlier chunks (Ids continue
// from it; it is advanced by this chunk's rows); offsetOut: write at out + rowBase rows instead of out.
bool LaunchSortFrames(const Workspace& ws, double* out, unsigned long long* rowBase, bool offsetOut, unsigned long long planeBase,
                      cudaStream_t st)
{
	static const bool configured = PTB_CUDA(cudaFuncSetAttribute(SortFrames, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                                                             static_cast<int>(kSortSmemBytes)));
	if (!configured) { return false; }
	SortFrames<<<ws.g.B, kSortThreads, kSortSmemBytes, st>>>(ws, out, rowBase, offsetOut ? 1 : 0, planeBase, ws.capRows);
	AdvanceRowBase<<<1, 1, 0, st>>>(ws, rowBase);
	CountLaunch(2);
	return PTB_LAUNCHED();
}

}  // namespace ptb
