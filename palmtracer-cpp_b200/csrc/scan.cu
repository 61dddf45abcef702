// Exclusive prefix sum of uint32 in place, with the element count either known on the host or read from device
// memory (so a chain of kernels needs no host round trip). data[n] receives the total; `total`, when given, too.
#include <algorithm>

#include "pt_common.cuh"

namespace ptb {

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t CountOf(const uint32_t* nptr, uint32_t nconst) { return nptr ? *nptr : nconst; }

// Block-wide exclusive scan of one value per thread; returns the block total in *total.
__device__ uint32_t BlockExclusive(uint32_t v, uint32_t* warpSums, uint32_t* total)
{
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	uint32_t x = v;
	#pragma unroll
	for (int d = 1; d < 32; d <<= 1) {
		const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
		if (lane >= d) { x += y; }
	}
	if (lane == 31) { warpSums[wid] = x; }
	__syncthreads();
	if (wid == 0) {
		uint32_t w = lane < (blockDim.x >> 5) ? warpSums[lane] : 0u;
		#pragma unroll
		for (int d = 1; d < 32; d <<= 1) {
			const uint32_t y = __shfl_up_sync(0xffffffffu, w, d);
			if (lane >= d) { w += y; }
		}
		warpSums[lane] = w;  // inclusive over warps
	}
	__syncthreads();
	const uint32_t warpBase = wid > 0 ? warpSums[wid - 1] : 0u;
	*total = warpSums[(blockDim.x >> 5) - 1];
	__syncthreads();
	return warpBase + x - v;
}

// One tile of kScanTile entries: exclusive scan in place, the tile's sum to blockSums[tile].
__device__ void ScanTile(uint32_t* data, uint32_t n, long long tile, uint32_t* warpSums, uint32_t* blockSums)
{
	const long long base = tile * kScanTile;
	uint32_t v[kScanItems];
	uint32_t sum = 0;
	#pragma unroll
	for (int k = 0; k < kScanItems; ++k) {
		const long long i = base + static_cast<long long>(threadIdx.x) * kScanItems + k;
		v[k] = i < n ? data[i] : 0u;
		sum += v[k];
	}
	uint32_t total;
	uint32_t off = BlockExclusive(sum, warpSums, &total);
	#pragma unroll
	for (int k = 0; k < kScanItems; ++k) {
		const long long i = base + static_cast<long long>(threadIdx.x) * kScanItems + k;
		if (i < n) { data[i] = off; }
		off += v[k];
	}
	if (threadIdx.x == 0) { blockSums[tile] = total; }
}

// Phase 1: local exclusive scan of each tile in place; tile sums to blockSums. Tiles are visited grid-stride, so the
// grid stays small when the device-side count is far below the capacity.
__global__ void __launch_bounds__(kScanThreads) ScanTiles(uint32_t* data, const uint32_t* nptr, uint32_t nconst,
                                                          uint32_t* blockSums)
{
	__shared__ uint32_t warpSums[32];
	const uint32_t n = CountOf(nptr, nconst);
	for (long long tile = blockIdx.x; tile * kScanTile < n; tile += gridDim.x) {
		ScanTile(data, n, tile, warpSums, blockSums);
	}
}


// Phase 2: one CTA scans the tile sums (exclusive) and stores the grand total.
__global__ void __launch_bounds__(kScanThreads) ScanSums(uint32_t* blockSums, const uint32_t* nptr, uint32_t nconst,
                                                         uint32_t* data, uint32_t* totalOut)
{
	__shared__ uint32_t warpSums[32];
	const uint32_t n = CountOf(nptr, nconst);
	const uint32_t tiles = static_cast<uint32_t>((static_cast<unsigned long long>(n) + kScanTile - 1) / kScanTile);
	uint32_t carry = 0;
	for (uint32_t base = 0; base < tiles; base += kScanThreads) {
		const uint32_t i = base + threadIdx.x;
		const uint32_t v = i < tiles ? blockSums[i] : 0u;
		uint32_t total;
		const uint32_t off = BlockExclusive(v, warpSums, &total);
		if (i < tiles) { blockSums[i] = carry + off; }
		carry += total;
	}
	if (threadIdx.x == 0) {
		data[n] = carry;
		if (totalOut) { *totalOut = carry; }
	}
}

// Phase 3: add the tile offsets.
__global__ void __launch_bounds__(kScanThreads) ScanAdd(uint32_t* data, const uint32_t* nptr, uint32_t nconst,
                                                        const uint32_t* blockSums)
{
	const uint32_t n = CountOf(nptr, nconst);
	for (long long tile = blockIdx.x; tile * kScanTile < n; tile += gridDim.x) {
		if (tile == 0) { continue; }
		const long long base = tile * kScanTile;
		const uint32_t add = blockSums[tile];
		#pragma unroll
		for (int k = 0; k < kScanItems; ++k) {
			const long long i = base + static_cast<long long>(k) * kScanThreads + threadIdx.x;
			if (i < n) { data[i] += add; }
		}
	}
}

}  // namespace

// `cap` bounds n (and sizes the grid); data must hold cap + 1 entries and blockSums cap / 4096 + 1.
bool ExclusiveScan(uint32_t* data, const uint32_t* nptr, uint32_t nconst, uint32_t cap, uint32_t* blockSums,
                   uint32_t* totalOut, cudaStream_t st)
{
	const uint32_t tiles = static_cast<uint32_t>((static_cast<unsigned long long>(cap) + kScanTile - 1) / kScanTile);
	const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(tiles, 2 * 148));
	ScanTiles<<<grid, kScanThreads, 0, st>>>(data, nptr, nconst, blockSums);
	ScanSums<<<1, kScanThreads, 0, st>>>(blockSums, nptr, nconst, data, totalOut);
	ScanAdd<<<grid, kScanThreads, 0, st>>>(data, nptr, nconst, blockSums);
	CountLaunch(3);
	return PTB_LAUNCHED();
}

}  // namespace ptb
