// Frame-to-frame tracking: greedy nearest-neighbour linking of localizations in consecutive planes.
//
// Reference: Tracks::Tracking (lib/tracking/Tracks.cpp:69-230, exported as Tracking, CPU/main.cpp:159-164):
//   1. points (Id, Plane, X, Y) ordered by (Plane, Id)                                     (loadPoints, :80-98)
//   2. for every pair of consecutive planes p, p + 1 that both hold points: all pairs within maxDistance,
//      d2 = dx * dx + dy * dy <= maxDistance^2, ordered by (d2, from, to)                   (getCandidates, :131-145;
//      track, :148-186)
//   3. in that order a pair links when its source has no successor and its target no predecessor yet
//   4. track numbers 1, 2, ... given to the chain heads in point order, then along each chain (:188-199)
//   5. output (Id, Track) per point in point order                                          (:203-212)
// On the GPU: the (Plane, Id) order is a counting sort by plane followed by a per-plane sort of (Id, input index).
// Step 2 does not test every pair: each plane is also sorted by X, and every point scans only the window of the next
// plane whose X lies within w of its own (binary search, then a forward scan), w slightly above maxDistance. A pair
// outside the window has fl(dx * dx) > maxDistance^2, so fl(fl(dx^2) + fl(dy^2)) > maxDistance^2 too (rounding is
// monotone) and the reference rejects it; inside, the reference's own test decides. Two passes, count then emit.
// Step 3 sorts each transition's pairs in one CTA and links them in order with one thread per transition
// (transitions touch disjoint successor and predecessor entries); step 4 is a scan over chain heads and pointer
// jumping along predecessor links. d2 is formed with explicitly rounded FP64 operations (no contraction), so the
// admitted pairs and their order are the reference's; ties in (Plane, Id), which the reference's unstable sort
// leaves unspecified, are ordered by input index.
#include <algorithm>
#include <cmath>
#include <vector>

#include "pt_common.cuh"

namespace ptb {

bool ExclusiveScan(uint32_t* data, const uint32_t* nptr, uint32_t nconst, uint32_t cap, uint32_t* blockSums,
                   uint32_t* totalOut, cudaStream_t st);

namespace {

constexpr uint32_t kNoLink = 0xffffffffu;
constexpr int kTrackThreads = 256;
constexpr int kSegSmem = 4096;  // pairs sorted in shared memory (64 KB); longer segments sort in global scratch
constexpr int kSortThreads = 512;

// static_cast<size_t>(double) of the reference for the values a localization table holds (non-negative integers)
__device__ __forceinline__ uint64_t ToIndex(double v) { return __double2ull_rz(v); }

__global__ void TrackKeys(const double* __restrict__ in, uint32_t n, uint64_t* plane, uint64_t* id, unsigned long long* minMax)
{
	unsigned long long lo = ~0ull, hi = 0ull;
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		const uint64_t p = ToIndex(in[4ull * i + 1]);
		plane[i] = p;
		id[i] = ToIndex(in[4ull * i]);
		lo = min(lo, static_cast<unsigned long long>(p));
		hi = max(hi, static_cast<unsigned long long>(p));
	}
	for (int d = 16; d > 0; d >>= 1) {
		lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, d));
		hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, d));
	}
	if ((threadIdx.x & 31) == 0) {
		atomicMin(&minMax[0], lo);
		atomicMax(&minMax[1], hi);
	}
}

__global__ void PlaneCount(const uint64_t* __restrict__ plane, uint32_t n, uint64_t minPlane, uint32_t* count)
{
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		atomicAdd(&count[plane[i] - minPlane], 1u);
	}
}

// Scatter point indices to their plane's range (arbitrary order inside a plane; the per-plane sort fixes it).
__global__ void PlaneScatter(const uint64_t* __restrict__ plane, const uint64_t* __restrict__ id, uint32_t n, uint64_t minPlane,
                             const uint32_t* __restrict__ begin, uint32_t* cursor, unsigned long long* k1, unsigned long long* k2)
{
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		const uint64_t p = plane[i] - minPlane;
		const uint32_t pos = begin[p] + atomicAdd(&cursor[p], 1u);
		k1[pos] = id[i];
		k2[pos] = i;
	}
}

__device__ __forceinline__ bool PairLess(unsigned long long a1, unsigned long long a2, unsigned long long b1, unsigned long long b2)
{
	return a1 < b1 || (a1 == b1 && a2 < b2);
}

// Bitonic sort of (k1, k2) pairs over a power-of-two length; entries past the segment hold the largest pair.
template <bool SMEM>
__device__ void BitonicPairs(unsigned long long* k1, unsigned long long* k2, uint32_t len)
{
	for (uint32_t size = 2; size <= len; size <<= 1) {
		for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
			for (uint32_t t = threadIdx.x; t < len / 2; t += blockDim.x) {
				const uint32_t lo = 2 * t - (t & (stride - 1));
				const uint32_t hi = lo + stride;
				const bool up = (lo & size) == 0;
				const bool swap = up ? PairLess(k1[hi], k2[hi], k1[lo], k2[lo]) : PairLess(k1[lo], k2[lo], k1[hi], k2[hi]);
				if (swap) {
					const unsigned long long a = k1[lo], b = k2[lo];
					k1[lo] = k1[hi]; k2[lo] = k2[hi];
					k1[hi] = a; k2[hi] = b;
				}
			}
			__syncthreads();
			if (!SMEM) { __threadfence_block(); }
		}
	}
}

// One CTA per segment [off[s], off[s + 1]): sorts its (k1, k2) pairs ascending. Segments longer than kSegSmem sort
// in global scratch at [2 off[s], 2 off[s] + 2 len) (a power of two below 2 len, so segments never overlap).
__global__ void __launch_bounds__(kSortThreads) SegmentSort(unsigned long long* k1, unsigned long long* k2, const uint32_t* __restrict__ off,
                                                            uint32_t nseg, unsigned long long* s1, unsigned long long* s2)
{
	extern __shared__ unsigned long long segSmem[];
	unsigned long long* a1 = segSmem;
	unsigned long long* a2 = segSmem + kSegSmem;
	for (uint32_t s = blockIdx.x; s < nseg; s += gridDim.x) {
		const uint32_t b = off[s], len = off[s + 1] - b;
		if (len <= 1) { continue; }
		uint32_t p2 = 1;
		while (p2 < len) { p2 <<= 1; }
		const bool smem = p2 <= static_cast<uint32_t>(kSegSmem);
		unsigned long long* x1 = smem ? a1 : s1 + 2ull * b;
		unsigned long long* x2 = smem ? a2 : s2 + 2ull * b;
		for (uint32_t i = threadIdx.x; i < p2; i += blockDim.x) {
			x1[i] = i < len ? k1[b + i] : ~0ull;
			x2[i] = i < len ? k2[b + i] : ~0ull;
		}
		__syncthreads();
		if (smem) { BitonicPairs<true>(x1, x2, p2); }
		else { BitonicPairs<false>(x1, x2, p2); }
		for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) {
			k1[b + i] = x1[i];
			k2[b + i] = x2[i];
		}
		__syncthreads();
	}
}

// Order-preserving map of a double to unsigned 64 bits (NaN, either sign, after +inf).
__device__ __forceinline__ unsigned long long XKey(double d)
{
	if (isnan(d)) { return ~0ull; }
	if (d == 0.0) { d = 0.0; }
	const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(d));
	return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

// Point order established: coordinates and plane of each ordered point, and the (X, point) pairs that the per-plane
// X sort orders.
__global__ void TrackGather(const double* __restrict__ in, const unsigned long long* __restrict__ src, const uint64_t* __restrict__ plane,
                            uint32_t n, uint64_t minPlane, double2* xy, uint32_t* rel, unsigned long long* xk1, unsigned long long* xk2)
{
	for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
		const uint32_t i = static_cast<uint32_t>(src[k]);
		const double x = in[4ull * i + 2];
		xy[k] = make_double2(x, in[4ull * i + 3]);
		rel[k] = static_cast<uint32_t>(plane[i] - minPlane);
		xk1[k] = XKey(x);
		xk2[k] = k;
	}
}

__device__ __forceinline__ double SqDistance(double2 a, double2 b)
{
	const double dx = __dsub_rn(a.x, b.x), dy = __dsub_rn(a.y, b.y);
	return __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
}

// One thread per point k: the points of the next plane inside its X window (all of them when the window is
// unbounded), tested with the reference's rule d2 <= r2. xs1/xs2: per plane, X keys ascending and their points.
// EMIT = false counts the admitted pairs of each point (count[k], and their total); EMIT = true writes them at their
// offsets as (d2 bits, source << 32 | target) — d2 >= 0, so its bits order like its value.
template <bool EMIT>
__global__ void __launch_bounds__(kTrackThreads) TrackPairs(const double2* __restrict__ xy, const uint32_t* __restrict__ rel,
                                                            const uint32_t* __restrict__ begin, const unsigned long long* __restrict__ xs1,
                                                            const unsigned long long* __restrict__ xs2, uint32_t n, uint32_t P, double r2,
                                                            double w, uint32_t* count, unsigned long long* total,
                                                            unsigned long long* k1, unsigned long long* k2)
{
	unsigned long long mine = 0;
	for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
		const uint32_t p = rel[k];
		if (p + 1 >= P) { continue; }
		uint32_t pos = begin[p + 1];
		const uint32_t c = begin[p + 2];
		const double2 me = xy[k];
		if (pos == c || isnan(me.x)) { continue; }  // a NaN coordinate admits no pair under any radius
		unsigned long long hiKey = ~0ull;
		if (w < __longlong_as_double(0x7ff0000000000000ll)) {
			// first X >= me.x - w, then forward while X <= me.x + w
			const unsigned long long loKey = XKey(me.x - w);
			hiKey = XKey(me.x + w);
			uint32_t lo = pos, hi = c;
			while (lo < hi) {
				const uint32_t mid = lo + ((hi - lo) >> 1);
				if (xs1[mid] < loKey) { lo = mid + 1; }
				else { hi = mid; }
			}
			pos = lo;
		}
		uint32_t found = 0;
		uint32_t at = EMIT ? count[k] : 0u;
		for (; pos < c && xs1[pos] <= hiKey; ++pos) {
			const uint32_t j = static_cast<uint32_t>(xs2[pos]);
			const double d2 = SqDistance(me, xy[j]);
			if (d2 <= r2) {
				if (EMIT) {
					k1[at] = static_cast<unsigned long long>(__double_as_longlong(d2));
					k2[at] = (static_cast<unsigned long long>(k) << 32) | j;
					++at;
				}
				++found;
			}
		}
		if (!EMIT) { count[k] = found; }
		mine += found;
	}
	if (!EMIT) {
		for (int d = 16; d > 0; d >>= 1) { mine += __shfl_xor_sync(0xffffffffu, mine, d); }
		if ((threadIdx.x & 31) == 0 && mine) { atomicAdd(total, mine); }
	}
}

// Pair ranges per transition: transition p owns the pairs of the points of plane p.
__global__ void TransitionOffsets(const uint32_t* __restrict__ begin, const uint32_t* __restrict__ pairBegin, uint32_t P, uint32_t* off)
{
	for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p <= P; p += gridDim.x * blockDim.x) { off[p] = pairBegin[begin[p]]; }
}

// One thread per transition: links its ordered pairs greedily (source without successor, target without
// predecessor). Transitions touch disjoint entries: successors of plane p, predecessors of plane p + 1.
__global__ void TrackLink(const unsigned long long* __restrict__ k2, const uint32_t* __restrict__ off, uint32_t P, uint32_t* next, uint32_t* prev)
{
	for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
		for (uint32_t c = off[p]; c < off[p + 1]; ++c) {
			const uint32_t from = static_cast<uint32_t>(k2[c] >> 32), to = static_cast<uint32_t>(k2[c] & 0xffffffffu);
			if (next[from] == kNoLink && prev[to] == kNoLink) {
				next[from] = to;
				prev[to] = from;
			}
		}
	}
}

__global__ void HeadFlags(const uint32_t* __restrict__ prev, uint32_t n, uint32_t* head, uint32_t* root)
{
	for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
		head[k] = prev[k] == kNoLink ? 1u : 0u;
		root[k] = prev[k] == kNoLink ? k : prev[k];
	}
}

// One pointer-jumping round: root[k] <- root[root[k]] (in place: a thread that reads an already advanced entry only
// moves further toward the chain head, so the rounds needed are at most those of the synchronous scheme).
__global__ void Jump(uint32_t* root, uint32_t n)
{
	for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) { root[k] = root[root[k]]; }
}

__global__ void TrackOutput(const unsigned long long* __restrict__ id, const uint32_t* __restrict__ root, const uint32_t* __restrict__ headRank,
                            uint32_t n, uint64_t* out)
{
	for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
		out[2ull * k] = id[k];
		out[2ull * k + 1] = static_cast<uint64_t>(headRank[root[k]]) + 1;
	}
}

constexpr size_t kSegSmemBytes = 2 * kSegSmem * sizeof(unsigned long long);

bool LaunchSegmentSort(unsigned long long* k1, unsigned long long* k2, const uint32_t* off, uint32_t nseg, unsigned long long* s1,
                       unsigned long long* s2, cudaStream_t st)
{
	static const bool configured = PTB_CUDA(cudaFuncSetAttribute(SegmentSort, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                                                             static_cast<int>(kSegSmemBytes)));
	if (!configured) { return false; }
	SegmentSort<<<std::max<uint32_t>(1, std::min<uint32_t>(nseg, 148u * 32)), kSortThreads, kSegSmemBytes, st>>>(k1, k2, off, nseg, s1, s2);
	CountLaunch();
	return PTB_LAUNCHED();
}

uint32_t Grid(uint64_t n, int threads) { return static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>((n + threads - 1) / threads, 148ull * 16))); }

}  // namespace

// dIn: device [n][4] (Id, Plane, X, Y); dOut: device [n][2] (Id, Track) in (Plane, Id) order. Synchronizes st (the
// plane range and the pair count size the buffers). Returns false with the error recorded.
bool TrackDevice(const double* dIn, uint64_t* dOut, uint64_t nPoints, double maxDistance, cudaStream_t st)
{
	if (nPoints == 0) { return true; }
	if (nPoints >= kNoLink) {
		SetError("Tracking: at most 2^32 - 2 points per call");
		return false;
	}
	const uint32_t n = static_cast<uint32_t>(nPoints);
	std::vector<void*> bufs;
	auto alloc = [&](auto*& p, size_t count) {
		using T = std::remove_pointer_t<std::remove_reference_t<decltype(p)>>;
		void* v = nullptr;
		const bool ok = PTB_CUDA(cudaMallocAsync(&v, std::max<size_t>(count, 1) * sizeof(T), st));
		p = static_cast<T*>(v);
		if (ok) { bufs.push_back(v); }
		return ok;
	};
	auto release = [&]() {
		for (void* b : bufs) { cudaFreeAsync(b, st); }
		bufs.clear();
	};
	const uint32_t G = Grid(n, kTrackThreads);
	uint64_t *plane = nullptr, *id = nullptr;
	unsigned long long* minMax = nullptr;
	unsigned long long hostMinMax[2] = {~0ull, 0ull};
	bool ok = alloc(plane, n) && alloc(id, n) && alloc(minMax, 3);
	ok = ok && PTB_CUDA(cudaMemcpyAsync(minMax, hostMinMax, sizeof(hostMinMax), cudaMemcpyHostToDevice, st));
	if (ok) {
		TrackKeys<<<G, kTrackThreads, 0, st>>>(dIn, n, plane, id, minMax);
		CountLaunch();
		ok = PTB_LAUNCHED();
	}
	ok = ok && PTB_CUDA(cudaMemcpyAsync(hostMinMax, minMax, sizeof(hostMinMax), cudaMemcpyDeviceToHost, st)) &&
	     PTB_CUDA(cudaStreamSynchronize(st));
	if (!ok) { release(); return false; }
	const uint64_t span = hostMinMax[1] - hostMinMax[0];
	if (span >= (1ull << 28)) {
		SetError("Tracking: planes span more than 2^28 values");
		release();
		return false;
	}
	const uint32_t P = static_cast<uint32_t>(span + 1);
	const uint64_t minPlane = hostMinMax[0];
	uint32_t *begin = nullptr, *cursor = nullptr, *scanScratch = nullptr;
	unsigned long long *pk1 = nullptr, *pk2 = nullptr, *s1 = nullptr, *s2 = nullptr;
	double2* xy = nullptr;
	uint32_t* rel = nullptr;
	unsigned long long *xk1 = nullptr, *xk2 = nullptr;
	const uint32_t scanCap = std::max(n, P) + 2;
	ok = alloc(begin, P + 2) && alloc(cursor, P) && alloc(scanScratch, scanCap / 4096 + 2) && alloc(pk1, n) && alloc(pk2, n) &&
	     alloc(s1, 2ull * n) && alloc(s2, 2ull * n) && alloc(xy, n) && alloc(rel, n) && alloc(xk1, n) && alloc(xk2, n);
	ok = ok && PTB_CUDA(cudaMemsetAsync(begin, 0, sizeof(uint32_t) * (P + 2), st)) &&
	     PTB_CUDA(cudaMemsetAsync(cursor, 0, sizeof(uint32_t) * P, st));
	if (ok) {
		// (Plane, Id) order: counting sort by plane, then (Id, input index) inside each plane
		PlaneCount<<<G, kTrackThreads, 0, st>>>(plane, n, minPlane, begin);
		CountLaunch();
		ok = PTB_LAUNCHED() && ExclusiveScan(begin, nullptr, P + 1, P + 1, scanScratch, nullptr, st);
	}
	if (ok) {
		PlaneScatter<<<G, kTrackThreads, 0, st>>>(plane, id, n, minPlane, begin, cursor, pk1, pk2);
		CountLaunch();
		ok = PTB_LAUNCHED() && LaunchSegmentSort(pk1, pk2, begin, P, s1, s2, st);
	}
	if (ok) {
		// coordinates in point order, then each plane's points by X for the window search
		TrackGather<<<G, kTrackThreads, 0, st>>>(dIn, pk2, plane, n, minPlane, xy, rel, xk1, xk2);
		CountLaunch();
		ok = PTB_LAUNCHED() && LaunchSegmentSort(xk1, xk2, begin, P, s1, s2, st);
	}
	// admitted pairs: count, offsets, emit
	uint32_t* pairBegin = nullptr;
	unsigned long long* total = nullptr;
	ok = ok && alloc(pairBegin, n + 2) && alloc(total, 1) && PTB_CUDA(cudaMemsetAsync(total, 0, sizeof(unsigned long long), st)) &&
	     PTB_CUDA(cudaMemsetAsync(pairBegin, 0, sizeof(uint32_t) * (n + 2), st));
	const double r2 = maxDistance * maxDistance;
	// X half-width of the search window: above sqrt(r2) by more than the rounding of dx, dx^2 and the bounds (and
	// above the largest |dx| whose square underflows to 0); unbounded when r2 is infinite or NaN
	const double w = std::isfinite(r2) ? std::max(std::sqrt(r2) * (1.0 + std::ldexp(1.0, -30)), 1e-150) : HUGE_VAL;
	if (ok) {
		TrackPairs<false><<<G, kTrackThreads, 0, st>>>(xy, rel, begin, xk1, xk2, n, P, r2, w, pairBegin, total, nullptr, nullptr);
		CountLaunch();
		ok = PTB_LAUNCHED();
	}
	unsigned long long pairs = 0;
	ok = ok && PTB_CUDA(cudaMemcpyAsync(&pairs, total, sizeof(pairs), cudaMemcpyDeviceToHost, st)) && PTB_CUDA(cudaStreamSynchronize(st));
	if (ok && pairs >= kNoLink) {
		SetError("Tracking: more than 2^32 - 2 candidate pairs (maxDistance too large for this density)");
		ok = false;
	}
	uint32_t *off = nullptr, *next = nullptr, *prev = nullptr, *head = nullptr, *root = nullptr;
	unsigned long long *ck1 = nullptr, *ck2 = nullptr, *c1 = nullptr, *c2 = nullptr;
	ok = ok && ExclusiveScan(pairBegin, nullptr, n, n + 1, scanScratch, nullptr, st);
	ok = ok && alloc(ck1, pairs) && alloc(ck2, pairs) && alloc(c1, 2 * pairs) && alloc(c2, 2 * pairs) && alloc(off, P + 1) &&
	     alloc(next, n) && alloc(prev, n) && alloc(head, n + 2) && alloc(root, n);
	if (ok && pairs > 0) {
		TrackPairs<true><<<G, kTrackThreads, 0, st>>>(xy, rel, begin, xk1, xk2, n, P, r2, w, pairBegin, nullptr, ck1, ck2);
		CountLaunch();
		ok = PTB_LAUNCHED();
	}
	ok = ok && PTB_CUDA(cudaMemsetAsync(next, 0xff, sizeof(uint32_t) * n, st)) && PTB_CUDA(cudaMemsetAsync(prev, 0xff, sizeof(uint32_t) * n, st));
	if (ok && pairs > 0) {
		TransitionOffsets<<<Grid(P + 1, kTrackThreads), kTrackThreads, 0, st>>>(begin, pairBegin, P, off);
		CountLaunch();
		ok = PTB_LAUNCHED() && LaunchSegmentSort(ck1, ck2, off, P, c1, c2, st);
	}
	if (ok && pairs > 0) {
		TrackLink<<<Grid(P, 128), 128, 0, st>>>(ck2, off, P, next, prev);
		CountLaunch();
		ok = PTB_LAUNCHED();
	}
	if (ok) {
		HeadFlags<<<G, kTrackThreads, 0, st>>>(prev, n, head, root);
		CountLaunch();
		ok = PTB_LAUNCHED() && ExclusiveScan(head, nullptr, n, n + 1, scanScratch, nullptr, st);
	}
	// a chain has at most one point per plane: ceil(log2(P)) + 1 rounds reach every head
	int rounds = 1;
	while ((1ull << (rounds - 1)) < P) { ++rounds; }
	for (int r = 0; ok && r < rounds; ++r) {
		Jump<<<G, kTrackThreads, 0, st>>>(root, n);
		CountLaunch();
		ok = PTB_LAUNCHED();
	}
	if (ok) {
		TrackOutput<<<G, kTrackThreads, 0, st>>>(pk1, root, head, n, dOut);
		CountLaunch();
		ok = PTB_LAUNCHED();
	}
	release();
	return ok;
}

}  // namespace ptb
