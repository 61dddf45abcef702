// Segmentation of the thresholded wavelet plane on the GPU: seeds, watershed, basin fusion, region statistics and
// the ordered candidate list. Reference: lib/localization/Segmentation2D.cpp (whole file) and SegmentationInfo.hpp.
//
// Data flow for one chunk of frames (global pixel index g = frame * N + y * W + x):
//   1. union-find connected components of the domain (8-connectivity) over the sparse domain list;
//   2. each seed (local maximum) inherits the label of its first raster-earlier seed neighbour, as getLocalMax()
//      does (Segmentation2D.cpp:309-327); root seeds are numbered in raster order through a per-row bitmask rank;
//   3. a component with one label is labelled directly; every other component (a "group") is flooded by one thread
//      (lane 0 of a warp that stages the group's box in shared memory; in strict mode a thread on global memory)
//      with a binary heap whose push/pop steps are those of libstdc++'s std::priority_queue, with the reference key
//      -v + pops * 1e-7 (Segmentation2D.cpp:336-385) and a pop counter local to the group. In strict mode a group is
//      a whole frame and the counter is frame-global, which is the reference's process exactly;
//   4. basin fusion (Segmentation2D.cpp:181-291) per group, then a second flood from one seed per basin;
//   5. exactness check of every per-component flood (below): a first test per boundary pair, then the rank test of
//      the pairs that fail it; a frame that fails both is flooded again per component with estimated frame-wide
//      aging and proven by a per-element test (the re-flood: shared-memory boxes, global memory for larger groups),
//      and a frame that fails that too is flooded again as one unit with the frame-global counter (the strict
//      process), so the labels always equal the reference's;
//   6. exact integer region sums (W1 is an integer in 2^-16 units) and the surf > 4 filter, in label order.
//
// Why a per-component flood equals the frame-wide one, and when it may not. Labels only spread inside a component,
// so a group's labels depend only on the order in which ITS pixels leave the heap; the frame-wide flood interleaves
// the other components' pops, which changes the aging term it * 1e-7 of the keys but nothing else. Every key of the
// frame-wide flood lies in [-v, -v + T * 1e-7], T = the frame's domain pixels (each is popped at most once). A
// flooded pixel N takes the label of whichever neighbour leaves the heap first. Let y be N's parent in the
// per-component flood and c the minimum W1 along y's parent chain down to its seed. If every element of that chain
// has a frame-wide key below the key of a competing neighbour z (another label), the chain is popped, element by
// element, before z can be: each element is pushed no later than its parent's pop and is then smaller than z. That
// holds when c - W1(z) > T * 1e-7. So if every flooded pixel N and every neighbour z of N with another label satisfy
// it, then (induction over the frame-wide flood's labelling order) every pixel receives its per-component label.
// In 2^-16 units the test is (c - W1(z)) * 152 > T (2^-16 / 152 exceeds 1e-7 by 4e-10 per pop, which covers the
// rounding of the FP64 keys, below 2e-11). About 4.5 % of the 1024 x 1024 benchmark frames have a pair failing it.
// Those pairs get the rank test (SuspectCheck), which bounds the two aging terms by the frame's pixel counts above
// and below the two W1 levels instead of by T; a frame failing that too is re-flooded (RefloodPlan .. RefloodBox)
// and, failing the re-flood's test, flooded again frame-wide. The rank test
// needs every pixel of the flood to be joined to a seed by a path that never falls below it, which holds for the
// first flood (every local maximum is a seed) but not for the second flood of a basin fusion (one seed per basin):
// there a pair failing the first test routes the frame directly.
#include "pt_common.cuh"

namespace ptb {

bool ExclusiveScan(uint32_t* data, const uint32_t* nptr, uint32_t nconst, uint32_t cap, uint32_t* blockSums,
                   uint32_t* totalOut, cudaStream_t st);

namespace {

constexpr int kThreads = 256;
constexpr int kGrid = 148 * 8;  // grid-stride kernels over device-side counts: 8 CTAs per SM

struct Pix {
	int f, y, x;
};

__device__ __forceinline__ Pix Decompose(uint32_t g, const Geometry& geo)
{
	Pix p;
	const uint32_t f = FastDivide(g, geo.divN);
	const uint32_t r = g - f * geo.divN.d;
	const uint32_t y = FastDivide(r, geo.divW);
	p.f = static_cast<int>(f);
	p.y = static_cast<int>(y);
	p.x = static_cast<int>(r - y * geo.divW.d);
	return p;
}

// Position of each predicated lane in a list grown by `counter`: one atomic per warp. Called by all 32 lanes.
__device__ __forceinline__ uint32_t WarpAppendIndex(bool pred, uint32_t* counter)
{
	const unsigned mask = __ballot_sync(0xffffffffu, pred);
	if (mask == 0) { return 0; }
	const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
	uint32_t base = 0;
	if (lane == leader) { base = atomicAdd(counter, static_cast<uint32_t>(__popc(mask))); }
	base = __shfl_sync(0xffffffffu, base, leader);
	return base + __popc(mask & ((1u << lane) - 1u));
}

// Sum of v over the run of consecutive lanes holding the same key as this lane, valid in the run's first lane
// (returned head = true); runs are maximal stretches of equal keys. Called by all 32 lanes.
template <typename T>
__device__ __forceinline__ T RunSum(uint32_t key, T v, bool& head)
{
	const int lane = threadIdx.x & 31;
	const uint32_t prev = __shfl_up_sync(0xffffffffu, key, 1);
	head = lane == 0 || prev != key;
	const unsigned heads = __ballot_sync(0xffffffffu, head);
	const unsigned after = lane == 31 ? 0u : (heads & (0xffffffffu << (lane + 1)));
	const int runEnd = after ? __ffs(after) - 2 : 31;
	#pragma unroll
	for (int d = 1; d < 32; d <<= 1) {
		const T t = __shfl_down_sync(0xffffffffu, v, d);
		if (lane + d <= runEnd) { v += t; }
	}
	return v;
}

__device__ __forceinline__ uint32_t Find(const uint32_t* par, uint32_t x)
{
	uint32_t p = __ldcg(par + x);
	while (p != x) {
		x = p;
		p = __ldcg(par + x);
	}
	return x;
}

// Union by smaller index; every root ends as the raster-first pixel of its component.
__device__ void Unite(uint32_t* par, uint32_t a, uint32_t b)
{
	for (;;) {
		a = Find(par, a);
		b = Find(par, b);
		if (a == b) { return; }
		if (a < b) {
			const uint32_t t = a;
			a = b;
			b = t;
		}
		const uint32_t old = atomicMin(par + a, b);
		if (old == a) { return; }
		a = old;
	}
}

// Component of a domain pixel once the components are enumerated; called only by kernels that do not write par, so
// its reads take the read-only cached path.
__device__ __forceinline__ uint32_t CompOf(const uint32_t* par, uint32_t p)
{
	const uint32_t x = __ldg(par + p);
	if (x & kCompTag) { return x & ~kCompTag; }
	return __ldg(par + x) & ~kCompTag;
}

// Component of domain pixel p once the roots carry their component ids (CompEnumerate): p's union-find chain walked
// to its tagged root through the SM's L1, and p then pointed at the root itself, as CompOf expects. While this runs a
// parent only ever changes to the root and the roots do not change, so a stale cached parent is still an ancestor
// and the walk still ends at the root; the pixels of a CTA mostly walk the same chains. A root left untagged (the
// component list overflowed; the chunk is redone) gives 0xffffffff.
__device__ __forceinline__ uint32_t CompWalk(uint32_t* par, uint32_t p)
{
	uint32_t x = p, v = __ldca(par + p);
	while (!(v & kCompTag) && v != x) {
		x = v;
		v = __ldca(par + x);
	}
	if (!(v & kCompTag)) { return 0xffffffffu; }
	if (x != p) { par[p] = x; }
	return v & ~kCompTag;
}

// 8-connectivity decision tree over the raster-earlier neighbours a = (y-1, x-1), b = (y-1, x), c = (y-1, x+1),
// d = (y, x-1): a pixel links to one of them at initialisation; only c together with a or d (b absent) joins two
// trees that are not yet known to touch, which is the single union left for CclUnion.
__device__ __forceinline__ void EarlierNeighbours(const Workspace& ws, uint32_t p, uint32_t& link, uint32_t& extra)
{
	const Pix q = Decompose(p, ws.g);
	const uint32_t W = static_cast<uint32_t>(ws.g.W);
	const bool up = q.y > 0, left = q.x > 0, right = q.x + 1 < ws.g.W;
	const bool a = up && left && (ws.code[p - W - 1] & kDomain);
	const bool b = up && (ws.code[p - W] & kDomain);
	const bool c = up && right && (ws.code[p - W + 1] & kDomain);
	const bool d = left && (ws.code[p - 1] & kDomain);
	link = p;
	extra = p;
	if (b) { link = p - W; }
	else if (c) {
		link = p - W + 1;
		if (a) { extra = p - W - 1; }
		else if (d) { extra = p - 1; }
	}
	else if (a) { link = p - W - 1; }
	else if (d) { link = p - 1; }
}

// Grid-stride loop in whole warps: every lane of a warp runs the same iterations (k may be >= n on the last one), so
// warp-wide collectives are safe inside.
#define PTB_WARP_LOOP(k, n)                                                                                        \
	for (uint32_t k##Base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u, k = k##Base + (threadIdx.x & 31u); \
	     k##Base < (n); k##Base += gridDim.x * blockDim.x, k = k##Base + (threadIdx.x & 31u))

// Links every domain pixel to one raster-earlier neighbour and lists the few that join two trees (most pixels have
// one raster-earlier link at most) for CclUnion, one atomic per warp. The list lives in lab, which nothing reads
// before the seed labels and the group scatter have written every domain pixel's label.
__global__ void CclInit(Workspace ws)
{
	const uint32_t n = min(ws.cnt->ndom, ws.capDom);
	const int lane = threadIdx.x & 31;
	PTB_WARP_LOOP(k, n)
	{
		uint32_t p = 0;
		bool join = false;
		if (k < n) {
			p = ws.dom[k];
			uint32_t link, extra;
			EarlierNeighbours(ws, p, link, extra);
			ws.par[p] = link;
			join = extra != p;
		}
		const unsigned m = __ballot_sync(0xffffffffu, join);
		if (m != 0u) {
			uint32_t at = 0;
			if (lane == 0) { at = atomicAdd(&ws.cnt->nunion, static_cast<uint32_t>(__popc(m))); }
			at = __shfl_sync(0xffffffffu, at, 0);
			if (join) { ws.lab[at + static_cast<uint32_t>(__popc(m & ((1u << lane) - 1u)))] = p; }
		}
	}
}

// The second union of the listed pixels (at most one per domain pixel, so the list fits lab).
__global__ void CclUnion(Workspace ws)
{
	const uint32_t n = ws.cnt->nunion;
	for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
		const uint32_t p = ws.lab[k];
		uint32_t link, extra;
		EarlierNeighbours(ws, p, link, extra);
		Unite(ws.par, p, extra);
	}
}

// Components: enumerate roots and tag par[root] with the component id.
// Component ids: one atomic per block and grid-stride step (roots are few, but a single counter hit by every warp
// serialises at the L2).
__global__ void __launch_bounds__(kThreads) CompEnumerate(Workspace ws)
{
	__shared__ uint32_t warpBase[kThreads / 32 + 1];
	const uint32_t n = min(ws.cnt->ndom, ws.capDom);
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
		const uint32_t k = base + threadIdx.x;
		uint32_t p = 0;
		bool root = false;
		if (k < n) {
			p = ws.dom[k];
			root = ws.par[p] == p;
		}
		const unsigned mask = __ballot_sync(0xffffffffu, root);
		if (lane == 0) { warpBase[warp] = __popc(mask); }
		__syncthreads();
		if (threadIdx.x == 0) {
			uint32_t total = 0;
			for (int w = 0; w < kThreads / 32; ++w) {
				const uint32_t c = warpBase[w];
				warpBase[w] = total;
				total += c;
			}
			warpBase[kThreads / 32] = total ? atomicAdd(&ws.cnt->ncomp, total) : 0u;
		}
		__syncthreads();
		const uint32_t c = warpBase[kThreads / 32] + warpBase[warp] + __popc(mask & ((1u << lane) - 1u));
		__syncthreads();  // warpBase is rewritten by the next step
		if (!root) { continue; }
		if (c >= ws.capComp) { atomicExch(&ws.cnt->overflow, 1u); continue; }
		ws.compRoot[c] = p;
		ws.compSize[c] = 0;
		ws.compNRoot[c] = 0;
		ws.compNSeed[c] = 0;
		ws.par[p] = c | kCompTag;
	}
}

__global__ void CompCount(Workspace ws)
{
	const uint32_t n = min(ws.cnt->ndom, ws.capDom);
	PTB_WARP_LOOP(k, n)
	{
		const uint32_t c = k < n ? CompWalk(ws.par, ws.dom[k]) : 0xffffffffu;
		bool head;
		const uint32_t count = RunSum<uint32_t>(c, 1u, head);
		if (head && c != 0xffffffffu) { atomicAdd(ws.compSize + c, count); }
	}
}

// Seed parents (Segmentation2D.cpp:309-327): first seed among (y-1,x-1), (y-1,x), (y-1,x+1), (y,x-1); none = root.
__global__ void SeedParent(Workspace ws)
{
	const uint32_t n = min(ws.cnt->nseed, ws.capSeed);
	const Geometry& geo = ws.g;
	for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
		const uint32_t s = ws.seeds[k];
		const Pix q = Decompose(s, geo);
		int dir = 0;
		if (q.y > 0) {
			const uint32_t up = s - static_cast<uint32_t>(geo.W);
			if (q.x > 0 && (ws.code[up - 1] & kSeed)) { dir = 1; }
			else if (ws.code[up] & kSeed) { dir = 2; }
			else if (q.x + 1 < geo.W && (ws.code[up + 1] & kSeed)) { dir = 3; }
		}
		if (dir == 0 && q.x > 0 && (ws.code[s - 1] & kSeed)) { dir = 4; }
		if (dir != 0) { ws.code[s] = static_cast<uint8_t>(ws.code[s] | (dir << kDirShift)); }
		else {
			const long long row = static_cast<long long>(q.f) * geo.H + q.y;
			atomicOr(ws.rootmask + row * geo.words + (q.x >> 5), 1u << (q.x & 31));
		}
	}
}

__global__ void RowCount(Workspace ws)
{
	const Geometry& geo = ws.g;
	const long long rows = static_cast<long long>(geo.B) * geo.H;
	for (long long r = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; r < rows; r += gridDim.x * static_cast<long long>(blockDim.x)) {
		uint32_t c = 0;
		const uint32_t* w = ws.rootmask + r * geo.words;
		for (int i = 0; i < geo.words; ++i) { c += __popc(w[i]); }
		ws.rowcnt[r] = c;
	}
}

__device__ __forceinline__ uint32_t SeedRoot(const Workspace& ws, uint32_t s)
{
	const uint32_t W = static_cast<uint32_t>(ws.g.W);
	for (;;) {
		const int dir = (ws.code[s] >> kDirShift) & 7;
		if (dir == 0) { return s; }
		s = dir == 1 ? s - W - 1 : dir == 2 ? s - W : dir == 3 ? s - W + 1 : s - 1;
	}
}

// Region id of a root seed: raster rank among root seeds of the chunk (frame-major, so labels follow raster order).
__device__ __forceinline__ uint32_t RegionOfRoot(const Workspace& ws, uint32_t rs)
{
	const Pix q = Decompose(rs, ws.g);
	const long long row = static_cast<long long>(q.f) * ws.g.H + q.y;
	const uint32_t* w = ws.rootmask + row * ws.g.words;
	uint32_t rank = ws.rowcnt[row];
	const int word = q.x >> 5;
	for (int i = 0; i < word; ++i) { rank += __popc(w[i]); }
	rank += __popc(w[word] & ((1u << (q.x & 31)) - 1u));
	return rank;
}

__global__ void SeedLabel(Workspace ws)
{
	const uint32_t n = min(ws.cnt->nseed, ws.capSeed);
	for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
		const uint32_t s = ws.seeds[k];
		const uint32_t rs = SeedRoot(ws, s);
		const uint32_t r = RegionOfRoot(ws, rs);
		if (r >= ws.capRegion) { atomicExch(&ws.cnt->overflow, 1u); continue; }
		ws.lab[s] = r + 1;
		const uint32_t c = CompOf(ws.par, s);
		atomicAdd(ws.compNSeed + c, 1u);
		if (rs == s) {
			ws.regCount[r] = 0;
			ws.regSumV[r] = 0;
			ws.regSumVJ[r] = 0;
			ws.regSumVI[r] = 0;
			ws.regFrame[r] = Decompose(s, ws.g).f;
			atomicAdd(ws.compNRoot + c, 1u);
			ws.compRegion[c] = r;
		}
	}
}

// Groups (fast mode): components with two or more regions. Sizes go to the offset arrays, scanned next.
__global__ void GroupEnumerate(Workspace ws)
{
	const uint32_t n = min(ws.cnt->ncomp, ws.capComp);
	PTB_WARP_LOOP(c, n)
	{
		const bool multi = c < n && ws.compNRoot[c] >= 2;
		const uint32_t m = WarpAppendIndex(multi, &ws.cnt->nmulti);
		if (!multi) { continue; }
		ws.multi[m] = c;
		ws.compRegion[c] = m;  // from here on: the group index of a multi-region component
		ws.gOff[m] = ws.compSize[c];
		ws.gSeedOff[m] = ws.compNSeed[c];
		ws.gRegOff[m] = ws.compNRoot[c];
		ws.gCurPix[m] = 0;
		ws.gCurSeed[m] = 0;
		ws.gCurReg[m] = 0;
	}
}

// Groups (strict mode): one per frame; sizes by atomics.
__global__ void GroupSizesStrict(Workspace ws)
{
	const uint32_t nd = min(ws.cnt->ndom, ws.capDom);
	for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nd; k += gridDim.x * blockDim.x) {
		atomicAdd(ws.gOff + Decompose(ws.dom[k], ws.g).f, 1u);
	}
	const uint32_t ns = min(ws.cnt->nseed, ws.capSeed);
	for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < ns; k += gridDim.x * blockDim.x) {
		const uint32_t s = ws.seeds[k];
		const int f = Decompose(s, ws.g).f;
		atomicAdd(ws.gSeedOff + f, 1u);
		if (((ws.code[s] >> kDirShift) & 7) == 0) { atomicAdd(ws.gRegOff + f, 1u); }
	}
}

// Frame-wide groups of the routed frames (one CTA): exclusive scans of their pixel, seed and region counts (zero for
// the frames that are not routed; the counts come from the detection kernel and the row scan of root seeds), cursors
// reset. Nothing to do when no frame is routed.
constexpr int kRedoThreads = 1024;

__global__ void __launch_bounds__(kRedoThreads) RedoOffsets(Workspace ws)
{
	__shared__ uint32_t warpSum[3][kRedoThreads / 32];
	__shared__ uint32_t carry[3];
	if (ws.cnt->nroute == 0) { return; }
	const int B = ws.g.B, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	if (threadIdx.x < 3) { carry[threadIdx.x] = 0; }
	__syncthreads();
	for (int base = 0; base <= B; base += kRedoThreads) {
		const int f = base + threadIdx.x;
		uint32_t v[3] = {0u, 0u, 0u};
		if (f < B && ws.frameRoute[f]) {
			v[0] = ws.frameDom[f];
			v[1] = ws.frameSeeds[f];
			v[2] = ws.rowcnt[static_cast<long long>(f + 1) * ws.g.H] - ws.rowcnt[static_cast<long long>(f) * ws.g.H];
		}
		uint32_t x[3];
		#pragma unroll
		for (int a = 0; a < 3; ++a) {
			x[a] = v[a];
			#pragma unroll
			for (int d = 1; d < 32; d <<= 1) {
				const uint32_t y = __shfl_up_sync(0xffffffffu, x[a], d);
				if (lane >= d) { x[a] += y; }
			}
			if (lane == 31) { warpSum[a][warp] = x[a]; }
		}
		__syncthreads();
		if (warp == 0) {
			#pragma unroll
			for (int a = 0; a < 3; ++a) {
				uint32_t w = warpSum[a][lane];
				#pragma unroll
				for (int d = 1; d < 32; d <<= 1) {
					const uint32_t y = __shfl_up_sync(0xffffffffu, w, d);
					if (lane >= d) { w += y; }
				}
				warpSum[a][lane] = w;  // inclusive over warps
			}
		}
		__syncthreads();
		if (f <= B) {
			uint32_t* out[3] = {ws.gOff, ws.gSeedOff, ws.gRegOff};
			#pragma unroll
			for (int a = 0; a < 3; ++a) {
				out[a][f] = carry[a] + (warp ? warpSum[a][warp - 1] : 0u) + x[a] - v[a];
			}
			ws.gCurPix[f] = 0;
			ws.gCurSeed[f] = 0;
			ws.gCurReg[f] = 0;
		}
		__syncthreads();
		if (threadIdx.x < 3) { carry[threadIdx.x] += warpSum[threadIdx.x][kRedoThreads / 32 - 1]; }
		__syncthreads();
	}
}

__device__ __forceinline__ int GroupOf(const Workspace& ws, uint32_t p, int strict)
{
	if (strict) { return Decompose(p, ws.g).f; }
	const uint32_t c = CompOf(ws.par, p);
	return ws.compNRoot[c] >= 2 ? static_cast<int>(ws.compRegion[c]) : -1;
}

// Domain pixels: labels of the non-seed pixels (single-region components take their region outright; flooded
// pixels of groups start unlabelled, seeds keep theirs) and the pixel lists of the groups. compRegion holds the
// region of a single-region component and the group index of a multi-region one.
// strict: 0 per-component groups, 1 every frame is a group, 2 only the frames routed to the frame-wide flood are
// (their seeds get their labels back, since a fusion may have cleared them; nothing to do when no frame is routed).
__global__ void GroupScatter(Workspace ws, int strict)
{
	if (strict == 2 && ws.cnt->nroute == 0) { return; }
	const uint32_t nd = min(ws.cnt->ndom, ws.capDom);
	const int lane = threadIdx.x & 31;
	PTB_WARP_LOOP(k, nd)
	{
		uint32_t p = 0;
		int m = -1;
		if (k < nd) {
			p = ws.dom[k];
			const bool seed = (ws.code[p] & kSeed) != 0;
			if (strict) {
				const int f = Decompose(p, ws.g).f;
				if (strict != 2 || ws.frameRoute[f] != 0) {
					if (!seed) { ws.lab[p] = 0u; }
					m = f;
				}
			}
			else {
				const uint32_t c = CompOf(ws.par, p);
				const uint32_t nroot = ws.compNRoot[c], r = ws.compRegion[c];
				if (!seed) { ws.lab[p] = nroot == 1 ? r + 1 : 0u; }
				m = nroot >= 2 ? static_cast<int>(r) : -1;
			}
		}
		// the group's pixel slots: one atomic per group and warp (consecutive domain pixels mostly share their group)
		const unsigned peers = __match_any_sync(0xffffffffu, m);
		const int leader = __ffs(peers) - 1;
		uint32_t at = 0;
		if (m >= 0 && lane == leader) { at = atomicAdd(ws.gCurPix + m, static_cast<uint32_t>(__popc(peers))); }
		at = __shfl_sync(0xffffffffu, at, leader) + static_cast<uint32_t>(__popc(peers & ((1u << lane) - 1u)));
		if (m >= 0) { ws.gPix[ws.gOff[m] + at] = p; }
	}
	const uint32_t ns = min(ws.cnt->nseed, ws.capSeed);
	for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < ns; k += gridDim.x * blockDim.x) {
		const uint32_t s = ws.seeds[k];
		const int m = GroupOf(ws, s, strict);
		if (m < 0) { continue; }
		if (strict == 2) {
			if (ws.frameRoute[m] == 0) { continue; }
			const uint32_t r = RegionOfRoot(ws, SeedRoot(ws, s));
			if (r < ws.capRegion) { ws.lab[s] = r + 1; }
		}
		ws.gSeed[ws.gSeedOff[m] + atomicAdd(ws.gCurSeed + m, 1u)] = s;
		if (((ws.code[s] >> kDirShift) & 7) == 0) { ws.gReg[ws.gRegOff[m] + atomicAdd(ws.gCurReg + m, 1u)] = ws.lab[s] - 1; }
	}
}

// In-place ascending heapsort of a small uint32 slice (one thread).
__device__ void SortSlice(uint32_t* a, uint32_t n)
{
	if (n < 2) { return; }
	auto sift = [a](uint32_t i, uint32_t len) {
		const uint32_t v = a[i];
		for (;;) {
			uint32_t c = 2 * i + 1;
			if (c >= len) { break; }
			if (c + 1 < len && a[c + 1] > a[c]) { ++c; }
			if (a[c] <= v) { break; }
			a[i] = a[c];
			i = c;
		}
		a[i] = v;
	};
	for (uint32_t i = n / 2; i-- > 0;) { sift(i, n); }
	for (uint32_t end = n - 1; end > 0; --end) {
		const uint32_t t = a[0];
		a[0] = a[end];
		a[end] = t;
		sift(0, end);
	}
}

// Binary heap with the steps of libstdc++'s push_heap / pop_heap (bits/stl_heap.h) under the reference comparator
// (Pixel::operator<, lib/Structs.hpp:20-27): "a before b" iff a.key > b.key, so the top holds the smallest key and
// equal keys come out in the same order as from the reference's std::priority_queue.
// Entry i lives at key[i * stride], pix[i * stride]: a lane-interleaved slice of shared memory while the heap holds at
// most `cap` entries, then (Spill) the group's own slice of global memory, sized for the whole group.
struct Heap {
	double* key;
	uint32_t* pix;
	uint32_t len;
	uint32_t stride;
	uint32_t cap;
	double* gkey;
	uint32_t* gpix;

	__device__ __forceinline__ static bool Less(double a, double b) { return a > b; }
	__device__ __forceinline__ double& K(uint32_t i) { return key[i * stride]; }
	__device__ __forceinline__ uint32_t& P(uint32_t i) { return pix[i * stride]; }

	__device__ void Spill()
	{
		for (uint32_t i = 0; i < len; ++i) {
			gkey[i] = K(i);
			gpix[i] = P(i);
		}
		key = gkey;
		pix = gpix;
		stride = 1;
		cap = 0xffffffffu;
	}

	__device__ void SiftUp(uint32_t hole, uint32_t top, double k, uint32_t v)
	{
		uint32_t parent = (hole - 1) / 2;
		while (hole > top && Less(K(parent), k)) {
			K(hole) = K(parent);
			P(hole) = P(parent);
			hole = parent;
			parent = (hole - 1) / 2;
		}
		K(hole) = k;
		P(hole) = v;
	}

	__device__ void Push(double k, uint32_t v)
	{
		if (len == cap) { Spill(); }
		const uint32_t hole = len++;
		if (hole == 0) { K(0) = k; P(0) = v; return; }
		SiftUp(hole, 0, k, v);
	}

	// Removes the top; returns its pixel.
	__device__ uint32_t Pop()
	{
		const uint32_t top = P(0);
		if (len > 1) {
			const uint32_t last = len - 1;  // element moved out of the way ("value" in __pop_heap)
			const double vk = K(last);
			const uint32_t vp = P(last);
			// __adjust_heap(first, 0, len = last, value)
			const uint32_t n = last;
			uint32_t hole = 0, child = 0;
			while (n >= 2 && child < (n - 1) / 2) {
				child = 2 * (child + 1);
				if (Less(K(child), K(child - 1))) { --child; }
				K(hole) = K(child);
				P(hole) = P(child);
				hole = child;
			}
			if ((n & 1) == 0 && child == (n - 2) / 2) {
				child = 2 * (child + 1);
				K(hole) = K(child - 1);
				P(hole) = P(child - 1);
				hole = child - 1;
			}
			if (hole == 0) { K(0) = vk; P(0) = vp; }
			else { SiftUp(hole, 0, vk, vp); }
		}
		--len;
		return top;
	}
};

constexpr int kFloodThreads = 64;
constexpr uint32_t kSmemHeap = 48;  // shared-memory heap entries per thread (12 bytes each)

struct FloodSmem {
	double key[kSmemHeap * kFloodThreads];
	uint32_t pix[kSmemHeap * kFloodThreads];
};

// The pixel data a flood reads and the labels it writes, in global memory (any group) ...
struct GlobalView {
	const Workspace& ws;
	__device__ __forceinline__ bool Dom(uint32_t p, int, int) const { return (__ldg(ws.code + p) & kDomain) != 0; }
	__device__ __forceinline__ uint32_t Lab(uint32_t p, int, int) const { return ws.lab[p]; }
	__device__ __forceinline__ void SetLab(uint32_t p, int, int, uint32_t v) const { ws.lab[p] = v; }
	__device__ __forceinline__ double W1(uint32_t p, int, int) const { return static_cast<double>(__ldg(ws.w1 + p)); }
	__device__ __forceinline__ uint32_t W1Fixed(uint32_t p, int, int) const { return __ldg(ws.w1 + p); }
	// parent-chain minimum of W1 (kNoChain on the flood's seeds), kept in par once the groups are scattered
	__device__ __forceinline__ uint32_t Chain(uint32_t p, int, int) const { return ws.par[p]; }
	__device__ __forceinline__ void SetChain(uint32_t p, int, int, uint32_t v) const { ws.par[p] = v; }
};

// ... or staged in shared memory: the group's bounding box with a one-pixel ring, row-major from (bx0, by0). Every
// pixel a flood of the group touches lies in it (a domain neighbour of a group pixel belongs to the group).
constexpr int kBoxCap = 320;          // staged pixels per group
constexpr uint32_t kBoxHeap = 64;     // shared-memory heap entries per group (12 bytes each)
constexpr int kBoxWarps = 8;          // groups (warps) per CTA

struct BoxSmem {
	double key[kBoxHeap];
	uint32_t pix[kBoxHeap];
	uint32_t w1[kBoxCap];     // W1 in 2^-16 units (0 < W1 < 2^32 on the domain)
	uint32_t lab[kBoxCap];
	uint32_t chain[kBoxCap];  // parent-chain minimum of W1 of the flooded pixels
	uint8_t flag[kBoxCap];    // bit 0: domain; bit 1: unlabelled when staged (the flood's labels are written back)
};

struct BoxView {
	BoxSmem& sm;
	int bx0, by0, bw;
	__device__ __forceinline__ int At(int y, int x) const { return (y - by0) * bw + (x - bx0); }
	__device__ __forceinline__ bool Dom(uint32_t, int y, int x) const { return (sm.flag[At(y, x)] & 1u) != 0; }
	__device__ __forceinline__ uint32_t Lab(uint32_t, int y, int x) const { return sm.lab[At(y, x)]; }
	__device__ __forceinline__ void SetLab(uint32_t, int y, int x, uint32_t v) const { sm.lab[At(y, x)] = v; }
	__device__ __forceinline__ double W1(uint32_t, int y, int x) const { return static_cast<double>(sm.w1[At(y, x)]); }
	__device__ __forceinline__ uint32_t W1Fixed(uint32_t, int y, int x) const { return sm.w1[At(y, x)]; }
	__device__ __forceinline__ uint32_t Chain(uint32_t, int y, int x) const { return sm.chain[At(y, x)]; }
	__device__ __forceinline__ void SetChain(uint32_t, int y, int x, uint32_t v) const { sm.chain[At(y, x)] = v; }
};

constexpr uint32_t kNoChain = 0xffffffffu;  // chain minimum of a flood's seeds (they were not pushed)

// The exactness test of one boundary pair: N (flooded, parent-chain minimum `chain`) against a neighbour of another
// label with W1 `w1z`, T = domain pixels of the frame (the bound of the frame-wide flood's pop counter).
__device__ __forceinline__ bool PairExact(uint32_t chain, uint32_t w1z, uint32_t T)
{
	return (static_cast<long long>(chain) - static_cast<long long>(w1z)) * 152 > static_cast<long long>(T);
}

// Marks frame f for the frame-wide flood (once).
__device__ __forceinline__ void RouteFrame(const Workspace& ws, int f, RouteReason why)
{
	if (atomicExch(ws.frameRoute + f, 1u) == 0u) {
		atomicAdd(&ws.cnt->nroute, 1u);
		atomicAdd(ws.cnt->routeWhy + why, 1u);
	}
}

// A boundary pair of frame f that failed the first test, kept for the rank test: the parent-chain minimum of the
// flooded pixel, W1 of the neighbour z of another label and W1 of z's highest domain neighbour (0 when z is a seed of
// the flood). Routes the frame, and returns false, when the list is full.
__device__ __forceinline__ bool SuspectPair(const Workspace& ws, int f, uint32_t chain, uint32_t w1z, uint32_t zmax)
{
	const uint32_t i = atomicAdd(&ws.cnt->nsuspect, 1u);
	if (i >= ws.capSuspect) {
		RouteFrame(ws, f, kRouteSuspectFull);
		return false;
	}
	ws.suspect[i] = make_uint4(static_cast<uint32_t>(f), chain, w1z, zmax);
	ws.frameSuspect[f] = 1u;
	return true;
}

// Highest W1 among the domain neighbours of pixel z (in global memory).
__device__ uint32_t HighestNeighbourGlobal(const Workspace& ws, uint32_t z)
{
	const Pix q = Decompose(z, ws.g);
	uint32_t best = 0;
	for (int dy = -1; dy <= 1; ++dy) {
		const int yy = q.y + dy;
		if (yy < 0 || yy >= ws.g.H) { continue; }
		for (int dx = -1; dx <= 1; ++dx) {
			const int xx = q.x + dx;
			if ((dx == 0 && dy == 0) || xx < 0 || xx >= ws.g.W) { continue; }
			const uint32_t nb = z + static_cast<uint32_t>(dy * ws.g.W + dx);
			if (__ldg(ws.code + nb) & kDomain) { best = max(best, __ldg(ws.w1 + nb)); }
		}
	}
	return best;
}

// Exactness test of a flooded pixel p of frame f against its 8 neighbours in global memory. A pair failing the first
// test is kept for the rank test (rank = true: a first flood, seeded at every local maximum) or routes the frame
// (rank = false: the second flood of a basin fusion, seeded at one maximum per basin, for which the rank bounds do
// not hold). Returns false when the frame was routed.
__device__ bool PixelExactGlobal(const Workspace& ws, uint32_t p, uint32_t T, int f, bool rank)
{
	const uint32_t chain = ws.par[p];
	if (chain == kNoChain) { return true; }
	const Pix q = Decompose(p, ws.g);
	const uint32_t L = ws.lab[p];
	for (int dy = -1; dy <= 1; ++dy) {
		const int yy = q.y + dy;
		if (yy < 0 || yy >= ws.g.H) { continue; }
		for (int dx = -1; dx <= 1; ++dx) {
			const int xx = q.x + dx;
			if ((dx == 0 && dy == 0) || xx < 0 || xx >= ws.g.W) { continue; }
			const uint32_t nb = p + static_cast<uint32_t>(dy * ws.g.W + dx);
			if (!(__ldg(ws.code + nb) & kDomain) || ws.lab[nb] == L) { continue; }
			const uint32_t w1z = __ldg(ws.w1 + nb);
			if (PairExact(chain, w1z, T)) { continue; }
			if (!rank) {
				RouteFrame(ws, f, kRouteFirstTest);
				return false;
			}
			// z pushed by the flood (a chain value) or one of its seeds
			const uint32_t zmax = ws.par[nb] == kNoChain ? 0u : HighestNeighbourGlobal(ws, nb);
			if (!SuspectPair(ws, f, chain, w1z, zmax)) { return false; }
		}
	}
	return true;
}

// Priority flood of one group from its labelled seeds (sorted ascending = raster order), Segmentation2D.cpp:336-385.
// kChain: record each pushed pixel's parent-chain minimum of W1 (the seeds must hold kNoChain) for the exactness test.
template <bool kChain, class View>
__device__ void FloodGroup(const Geometry& geo, const View& v, const uint32_t* seedList, uint32_t nSeeds, Heap& heap)
{
	for (uint32_t i = 0; i < nSeeds; ++i) {
		const uint32_t s = seedList[i];
		const Pix q = Decompose(s, geo);
		bool open = false;
		for (int dy = -1; dy <= 1 && !open; ++dy) {
			const int yy = q.y + dy;
			if (yy < 0 || yy >= geo.H) { continue; }
			for (int dx = -1; dx <= 1 && !open; ++dx) {
				const int xx = q.x + dx;
				if ((dx == 0 && dy == 0) || xx < 0 || xx >= geo.W) { continue; }
				const uint32_t nb = s + static_cast<uint32_t>(dy * geo.W + dx);
				if (!v.Dom(nb, yy, xx) || v.Lab(nb, yy, xx) == 0) { open = true; }
			}
		}
		if (open) { heap.Push(-(v.W1(s, q.y, q.x) * kW1Unit), s); }
	}
	unsigned long long pops = 0;
	while (heap.len > 0) {
		const uint32_t p = heap.Pop();
		++pops;
		const Pix q = Decompose(p, geo);
		const uint32_t L = v.Lab(p, q.y, q.x);
		// the 8 neighbours in the reference's scan order; their domain flag, label and W1 are loaded together (each
		// neighbour's label is written at most once below, after its own test)
		uint32_t nb[8];
		int ny[8], nx[8];
		bool in[8], dm[8];
		uint32_t lb[8];
		double wv[8];
		#pragma unroll
		for (int t = 0; t < 8; ++t) {
			const int dy = t < 3 ? -1 : (t < 5 ? 0 : 1);
			const int dx = t < 3 ? t - 1 : (t < 5 ? (t == 3 ? -1 : 1) : t - 6);
			ny[t] = q.y + dy;
			nx[t] = q.x + dx;
			in[t] = ny[t] >= 0 && ny[t] < geo.H && nx[t] >= 0 && nx[t] < geo.W;
			nb[t] = p + static_cast<uint32_t>(dy * geo.W + dx);
		}
		#pragma unroll
		for (int t = 0; t < 8; ++t) {
			dm[t] = in[t] && v.Dom(nb[t], ny[t], nx[t]);
			lb[t] = dm[t] ? v.Lab(nb[t], ny[t], nx[t]) : 1u;
			wv[t] = dm[t] ? v.W1(nb[t], ny[t], nx[t]) : 0.0;
		}
		const double age = __dmul_rn(static_cast<double>(pops), kEps);
		const uint32_t chain = kChain ? min(v.Chain(p, q.y, q.x), v.W1Fixed(p, q.y, q.x)) : 0u;
		#pragma unroll
		for (int t = 0; t < 8; ++t) {
			if (dm[t] && lb[t] == 0) {
				// key = -v + it * EPSILON, both operations rounded separately as in the reference
				const double k = __dadd_rn(-(wv[t] * kW1Unit), age);
				heap.Push(k, nb[t]);
				v.SetLab(nb[t], ny[t], nx[t], L);
				if (kChain) { v.SetChain(nb[t], ny[t], nx[t], chain); }
			}
		}
	}
}

// Flood with the heap in this thread's shared-memory slice, moving to the group's global slice (hk, hp) if it outgrows it.
template <bool kChain>
__device__ void FloodGroupGlobal(const Workspace& ws, const uint32_t* seedList, uint32_t nSeeds, double* hk, uint32_t* hp,
                                 FloodSmem& sm)
{
	Heap heap{sm.key + threadIdx.x, sm.pix + threadIdx.x, 0, kFloodThreads, kSmemHeap, hk, hp};
	FloodGroup<kChain>(ws.g, GlobalView{ws}, seedList, nSeeds, heap);
}

// Frame-wide floods (groups = frames): every frame (strict mode) or only the frames that failed the exactness test of
// their per-component floods (routed: nothing to do when no frame did).
__global__ void __launch_bounds__(kFloodThreads) GroupFlood(Workspace ws, uint32_t nGroupsStrict, int routed)
{
	__shared__ FloodSmem sm;
	if (routed && ws.cnt->nroute == 0) { return; }
	const uint32_t n = nGroupsStrict ? nGroupsStrict : ws.cnt->nmulti;
	for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
		if (routed && ws.frameRoute[m] == 0) { continue; }
		const uint32_t nSeeds = ws.gSeedOff[m + 1] - ws.gSeedOff[m];
		uint32_t* seeds = ws.gSeed + ws.gSeedOff[m];
		SortSlice(seeds, nSeeds);
		FloodGroupGlobal<false>(ws, seeds, nSeeds, ws.heapKey + ws.gOff[m], ws.heapPix + ws.gOff[m], sm);
	}
}

// One warp per group (groups are components, never whole frames): the lanes stage the group's bounding box with a
// one-pixel ring in shared memory, lane 0 floods it there (the flood is one serial chain of heap operations; with
// the box in shared memory each of its steps waits on shared memory instead of on L2 or DRAM), and the lanes write
// back the labels the flood set. A group whose box exceeds kBoxCap pixels is flooded in global memory by lane 0.
// rank: pairs failing the first exactness test are kept for the rank test (else they route the frame directly).
__global__ void __launch_bounds__(kBoxWarps * 32) GroupFloodBox(Workspace ws, int rank)
{
	__shared__ BoxSmem boxes[kBoxWarps];
	BoxSmem& sm = boxes[threadIdx.x / 32];
	const int lane = threadIdx.x & 31;
	const Geometry& geo = ws.g;
	const uint32_t n = ws.cnt->nmulti;
	// each warp takes the next group from a work queue when its previous one is done: group floods vary in length,
	// and the CTAs beyond the resident ones (the box staging limits an SM to a few) find little left
	for (;;) {
		uint32_t m = 0;
		if (lane == 0) { m = atomicAdd(&ws.cnt->boxNext, 1u); }
		m = __shfl_sync(0xffffffffu, m, 0);
		if (m >= n) { break; }
		const uint32_t off = ws.gOff[m], nPix = ws.gOff[m + 1] - off;
		const uint32_t nSeeds = ws.gSeedOff[m + 1] - ws.gSeedOff[m];
		uint32_t* seeds = ws.gSeed + ws.gSeedOff[m];
		int x0 = geo.W, y0 = geo.H, x1 = -1, y1 = -1, f = 0;
		for (uint32_t i = lane; i < nPix; i += 32) {
			const Pix q = Decompose(ws.gPix[off + i], geo);
			x0 = min(x0, q.x); x1 = max(x1, q.x); y0 = min(y0, q.y); y1 = max(y1, q.y);
			f = q.f;
		}
		#pragma unroll
		for (int d = 16; d > 0; d >>= 1) {
			x0 = min(x0, __shfl_xor_sync(0xffffffffu, x0, d));
			y0 = min(y0, __shfl_xor_sync(0xffffffffu, y0, d));
			x1 = max(x1, __shfl_xor_sync(0xffffffffu, x1, d));
			y1 = max(y1, __shfl_xor_sync(0xffffffffu, y1, d));
		}
		f = __shfl_sync(0xffffffffu, f, 0);  // lane 0 holds the group's first pixel (a group has at least two)
		const int bx0 = max(x0 - 1, 0), by0 = max(y0 - 1, 0);
		const int bw = min(x1 + 1, geo.W - 1) - bx0 + 1, bh = min(y1 + 1, geo.H - 1) - by0 + 1;
		double* hk = ws.heapKey + off;
		uint32_t* hp = ws.heapPix + off;
		const uint32_t T = ws.frameDom[f];
		if (nPix == 0 || bw * bh > kBoxCap) {
			for (uint32_t i = lane; i < nPix; i += 32) { ws.par[ws.gPix[off + i]] = kNoChain; }
			__syncwarp();
			if (lane == 0 && nPix > 0) {
				SortSlice(seeds, nSeeds);
				Heap heap{sm.key, sm.pix, 0, 1, kBoxHeap, hk, hp};
				FloodGroup<true>(geo, GlobalView{ws}, seeds, nSeeds, heap);
			}
			__syncwarp();
			bool exact = true;
			for (uint32_t i = lane; i < nPix && exact; i += 32) { exact = PixelExactGlobal(ws, ws.gPix[off + i], T, f, rank != 0); }
			continue;
		}
		const uint32_t base = static_cast<uint32_t>(f) * static_cast<uint32_t>(geo.N) + static_cast<uint32_t>(by0 * geo.W + bx0);
		for (int i = lane; i < bw * bh; i += 32) {
			const int r = i / bw, c = i - r * bw;
			const uint32_t p = base + static_cast<uint32_t>(r * geo.W + c);
			const bool dom = (__ldg(ws.code + p) & kDomain) != 0;
			const uint32_t lb = dom ? ws.lab[p] : 0u;
			sm.w1[i] = dom ? __ldg(ws.w1 + p) : 0u;
			sm.lab[i] = lb;
			sm.chain[i] = kNoChain;
			sm.flag[i] = static_cast<uint8_t>((dom ? 1u : 0u) | (dom && lb == 0 ? 2u : 0u));
		}
		__syncwarp();
		if (lane == 0) {
			SortSlice(seeds, nSeeds);
			Heap heap{sm.key, sm.pix, 0, 1, kBoxHeap, hk, hp};
			FloodGroup<true>(geo, BoxView{sm, bx0, by0, bw}, seeds, nSeeds, heap);
		}
		__syncwarp();
		for (int i = lane; i < bw * bh; i += 32) {
			if (!(sm.flag[i] & 2u) || sm.lab[i] == 0) { continue; }
			const int r = i / bw, c = i - r * bw;
			ws.lab[base + static_cast<uint32_t>(r * geo.W + c)] = sm.lab[i];
			// exactness test against the neighbours of other labels (every neighbour in the frame lies in the box); a
			// pair failing the first test is kept for the rank test
			const uint32_t L = sm.lab[i], chain = sm.chain[i];
			for (int dy = -1; dy <= 1; ++dy) {
				if (r + dy < 0 || r + dy >= bh) { continue; }
				for (int dx = -1; dx <= 1; ++dx) {
					if ((dx == 0 && dy == 0) || c + dx < 0 || c + dx >= bw) { continue; }
					const int j = i + dy * bw + dx;
					if (!(sm.flag[j] & 1u) || sm.lab[j] == L || PairExact(chain, sm.w1[j], T)) { continue; }
					if (!rank) {
						RouteFrame(ws, f, kRouteFirstTest);
						continue;
					}
					// z = pixel j is a group pixel, so its neighbours in the frame lie in the box as well
					uint32_t zmax = 0;
					if (sm.chain[j] != kNoChain) {
						const int zr = r + dy, zc = c + dx;
						for (int ey = -1; ey <= 1; ++ey) {
							if (zr + ey < 0 || zr + ey >= bh) { continue; }
							for (int ex = -1; ex <= 1; ++ex) {
								if ((ex == 0 && ey == 0) || zc + ex < 0 || zc + ex >= bw) { continue; }
								zmax = max(zmax, sm.w1[j + ey * bw + ex]);  // 0 off the domain
							}
						}
					}
					SuspectPair(ws, f, chain, sm.w1[j], zmax);
				}
			}
		}
		__syncwarp();
	}
}

// Basin fusion of one group (Segmentation2D.cpp:181-291) followed by the reseeded second flood.
// Groups: the per-component groups (nGroupsStrict = 0; the second flood is checked for exactness), every frame
// (strict mode) or only the frames flooded again frame-wide (routed).
__global__ void __launch_bounds__(kFloodThreads) GroupFuse(Workspace ws, uint32_t nGroupsStrict, double ratio, int routed)
{
	__shared__ FloodSmem sm;
	if (routed && ws.cnt->nroute == 0) { return; }
	const uint32_t n = nGroupsStrict ? nGroupsStrict : ws.cnt->nmulti;
	const Geometry& geo = ws.g;
	for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
		if (routed && ws.frameRoute[m] == 0) { continue; }
		uint32_t* regs = ws.gReg + ws.gRegOff[m];
		uint32_t nReg = ws.gRegOff[m + 1] - ws.gRegOff[m];
		const uint32_t* pix = ws.gPix + ws.gOff[m];
		const uint32_t nPix = ws.gOff[m + 1] - ws.gOff[m];
		if (nReg == 0) { continue; }
		SortSlice(regs, nReg);  // label order
		// every pass that changes something removes at least one basin, so nReg + 1 passes always reach a stable state
		const uint32_t passes = nReg + 1;
		for (uint32_t iter = 0; iter < passes; ++iter) {
			for (uint32_t i = 0; i < nReg; ++i) {
				const uint32_t r = regs[i];
				ws.fuMaxWN[r] = -1e10;
				ws.fuMinP[r] = 1e10;
				ws.fuMaxP[r] = -1e10;
				ws.fuMaxPos[r] = 0xffffffffu;
				ws.fuWNPos[r] = 0xffffffffu;
				ws.fuNeighbour[r] = 0;
				ws.fuLocked[r] = 0;
				ws.fuBecome[r] = r;
			}
			for (uint32_t i = 0; i < nPix; ++i) {
				const uint32_t p = pix[i];
				const uint32_t L = ws.lab[p];
				if (L == 0) { continue; }
				const uint32_t r = L - 1;
				const double v = static_cast<double>(ws.w1[p]) * kW1Unit;
				ws.fuMinP[r] = fmin(ws.fuMinP[r], v);
				// first raster pixel reaching the maximum (strict > in raster order)
				if (v > ws.fuMaxP[r] || (v == ws.fuMaxP[r] && p < ws.fuMaxPos[r])) {
					ws.fuMaxP[r] = v;
					ws.fuMaxPos[r] = p;
				}
				// strongest boundary pixel; its first differently-labelled neighbour in 3x3 scan order
				const Pix q = Decompose(p, geo);
				uint32_t other = 0;
				for (int dy = -1; dy <= 1 && other == 0; ++dy) {
					const int yy = q.y + dy;
					if (yy < 0 || yy >= geo.H) { continue; }
					for (int dx = -1; dx <= 1 && other == 0; ++dx) {
						const int xx = q.x + dx;
						if ((dx == 0 && dy == 0) || xx < 0 || xx >= geo.W) { continue; }
						const uint32_t nb = p + static_cast<uint32_t>(dy * geo.W + dx);
						if (!(ws.code[nb] & kDomain)) { continue; }
						const uint32_t nl = ws.lab[nb];
						if (nl != 0 && nl != L) { other = nl; }
					}
				}
				if (other != 0 && (v > ws.fuMaxWN[r] || (v == ws.fuMaxWN[r] && p < ws.fuWNPos[r]))) {
					ws.fuMaxWN[r] = v;
					ws.fuWNPos[r] = p;
					ws.fuNeighbour[r] = other;
				}
			}
			bool change = false;
			for (uint32_t i = 0; i < nReg; ++i) {
				const uint32_t r = regs[i];
				if (ws.fuNeighbour[r] == 0) { continue; }
				const uint32_t nb = ws.fuNeighbour[r] - 1;
				if (ws.fuLocked[r] || ws.fuLocked[nb]) { continue; }
				const double delta = ws.fuMaxP[r] - ws.fuMinP[r];
				if (fabs(delta) <= 2.220446049250313e-16) { continue; }
				const double rr = (ws.fuMaxP[r] - ws.fuMaxWN[r]) / delta;
				if (rr < ratio && ws.fuMaxP[r] < ws.fuMaxP[nb]) {
					ws.fuBecome[r] = nb;
					ws.fuLocked[nb] = 1;
					ws.fuLocked[r] = 1;
					change = true;
				}
			}
			if (!change) { break; }
			for (uint32_t i = 0; i < nPix; ++i) {
				const uint32_t p = pix[i];
				const uint32_t L = ws.lab[p];
				if (L != 0) { ws.lab[p] = ws.fuBecome[L - 1] + 1; }
			}
			uint32_t kept = 0;
			for (uint32_t i = 0; i < nReg; ++i) {
				if (ws.fuBecome[regs[i]] == regs[i]) { regs[kept++] = regs[i]; }
			}
			nReg = kept;
		}
		// one seed per basin at its first maximum, then flood again
		const bool check = nGroupsStrict == 0;
		for (uint32_t i = 0; i < nPix; ++i) {
			ws.lab[pix[i]] = 0;
			if (check) { ws.par[pix[i]] = kNoChain; }
		}
		uint32_t* seeds = ws.gSeed + ws.gSeedOff[m];  // reuse the seed slice (nReg <= number of seeds)
		for (uint32_t i = 0; i < nReg; ++i) {
			const uint32_t r = regs[i];
			seeds[i] = ws.fuMaxPos[r];
			ws.lab[ws.fuMaxPos[r]] = r + 1;
		}
		SortSlice(seeds, nReg);
		if (!check) {
			FloodGroupGlobal<false>(ws, seeds, nReg, ws.heapKey + ws.gOff[m], ws.heapPix + ws.gOff[m], sm);
			continue;
		}
		FloodGroupGlobal<true>(ws, seeds, nReg, ws.heapKey + ws.gOff[m], ws.heapPix + ws.gOff[m], sm);
		const int f = Decompose(pix[0], geo).f;
		const uint32_t T = ws.frameDom[f];
		for (uint32_t i = 0; i < nPix; ++i) {
			if (!PixelExactGlobal(ws, pix[i], T, f, false)) { break; }
		}
	}
}

// ---- Rank test of the per-component floods ---------------------------------------------------------------------
// The frame-wide flood pops in W1 order up to its aging term: a pixel whose W1 exceeds another's by more than
// delta = T * 1e-7 (the largest aging term, T = the frame's domain pixels) leaves the heap first, since the path that
// joins it to its component's maximum (a seed) never falls below its W1 and some pixel of that path is always in the
// heap. So a pixel p is popped at a position g(p) <= B(p) = #{domain pixels with W1 >= W1(p) - delta} and its pushes
// age by g(p) * 1e-7, while a pixel n is popped at g(n) > #{poppable pixels with W1 > W1(n) + delta}. For a pair
// with parent-chain minimum c (every chain element has W1 >= c and was pushed by a chain element, so with aging at
// most B_c * 1e-7, B_c = #{W1 >= c - delta}) and competing neighbour z (pushed by one of its neighbours, none higher
// than zmax, so with aging at least A_z * 1e-7, A_z = #{poppable W1 > zmax + delta} + 1; 0 when z is a seed), every
// chain element leaves the frame-wide heap before z when
//   (c - W1(z)) * 2^-16 > (B_c - A_z + 1) * 1e-7,   i.e. (c - W1(z)) * 78125 > (B_c - A_z + 1) * 512,
// the + 1 covering the rounding of the FP64 keys. The counts are exact: SuspectCount compares every domain pixel of
// the frame with the pair's two levels. A pair failing this too routes its frame to the frame-wide flood.

constexpr int kPlanThreads = 1024;

// Step 1 (one CTA): a slot for each frame with pairs kept for the rank test, in frame order (frameSuspect[f] =
// slot + 1), and the pairs ordered by slot with zeroed counts. Frames beyond kRankSlots slots or with more than
// kPairsPerFrame pairs are routed instead (and get no slot). Nothing to do without such pairs.
__global__ void __launch_bounds__(kPlanThreads) SuspectPlan(Workspace ws)
{
	__shared__ uint32_t warpSum[kPlanThreads / 32];
	__shared__ uint32_t carry;
	__shared__ uint32_t slotCount[kRankSlots], slotCur[kRankSlots];
	if (ws.cnt->nsuspect == 0) { return; }
	const int B = ws.g.B, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	if (threadIdx.x == 0) { carry = 0; }
	if (threadIdx.x < kRankSlots) { slotCount[threadIdx.x] = 0; }
	__syncthreads();
	for (int base = 0; base < B; base += kPlanThreads) {
		const int f = base + static_cast<int>(threadIdx.x);
		const uint32_t v = (f < B && ws.frameSuspect[f] != 0u) ? 1u : 0u;
		uint32_t x = v;
		#pragma unroll
		for (int d = 1; d < 32; d <<= 1) {
			const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
			if (lane >= d) { x += y; }
		}
		if (lane == 31) { warpSum[warp] = x; }
		__syncthreads();
		if (warp == 0) {
			uint32_t w = warpSum[lane];
			#pragma unroll
			for (int d = 1; d < 32; d <<= 1) {
				const uint32_t y = __shfl_up_sync(0xffffffffu, w, d);
				if (lane >= d) { w += y; }
			}
			warpSum[lane] = w;
		}
		__syncthreads();
		if (v) {
			const uint32_t slot = carry + (warp ? warpSum[warp - 1] : 0u) + x - 1u;
			if (slot < kRankSlots) { ws.frameSuspect[f] = slot + 1u; }
			else {
				ws.frameSuspect[f] = 0u;
				RouteFrame(ws, f, kRouteRankSlots);
			}
		}
		__syncthreads();
		if (threadIdx.x == 0) { carry += warpSum[kPlanThreads / 32 - 1]; }
		__syncthreads();
	}
	if (threadIdx.x == 0) { ws.cnt->nslots = carry; }
	const uint32_t nrec = min(ws.cnt->nsuspect, ws.capSuspect);
	for (uint32_t i = threadIdx.x; i < nrec; i += kPlanThreads) {
		const uint32_t s = ws.frameSuspect[ws.suspect[i].x];
		if (s != 0u) { atomicAdd(slotCount + (s - 1u), 1u); }
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		uint32_t off = 0;
		for (uint32_t k = 0; k < kRankSlots; ++k) {
			ws.rankSlotOff[k] = off;
			slotCur[k] = off;
			off += slotCount[k];
		}
		ws.rankSlotOff[kRankSlots] = off;
	}
	__syncthreads();
	for (uint32_t i = threadIdx.x; i < nrec; i += kPlanThreads) {
		const uint32_t f = ws.suspect[i].x, s = ws.frameSuspect[f];
		if (s == 0u) { continue; }
		ws.rankOrder[atomicAdd(slotCur + (s - 1u), 1u)] = i;
		ws.rankCount[2 * i] = 0u;
		ws.rankCount[2 * i + 1] = 0u;
	}
	__syncthreads();
	// frames with too many pairs: routed; their slots stay empty in the counting pass (frameSuspect = 0)
	for (uint32_t i = threadIdx.x; i < nrec; i += kPlanThreads) {
		const uint32_t f = ws.suspect[i].x, s = ws.frameSuspect[f];
		if (s != 0u && slotCount[s - 1u] > kPairsPerFrame) { RouteFrame(ws, static_cast<int>(f), kRoutePairs); }
	}
	__syncthreads();
	for (int f = threadIdx.x; f < B; f += kPlanThreads) {
		const uint32_t s = ws.frameSuspect[f];
		if (s != 0u && slotCount[s - 1u] > kPairsPerFrame) { ws.frameSuspect[f] = 0u; }
	}
}

// The two levels of pair i of frame f: B_c counts W1 >= lowB, A_z counts poppable W1 > lowA (lowA = 2^32 - 1 when
// there is nothing to count: z a seed, or a level beyond the W1 range).
__device__ __forceinline__ void PairLevels(const Workspace& ws, const uint4& r, uint32_t& lowB, uint32_t& lowA)
{
	const uint32_t T = ws.frameDom[r.x];
	const uint32_t delta = static_cast<uint32_t>((static_cast<unsigned long long>(T) * 65536ull) / 10000000ull) + 1u;
	lowB = r.y > delta ? r.y - delta : 0u;
	const unsigned long long a = static_cast<unsigned long long>(r.w) + delta;
	lowA = (r.w == 0u || a >= 0xffffffffull) ? 0xffffffffu : static_cast<uint32_t>(a);
}

// Step 2: exact counts of every pair's two levels over its frame's domain pixels, one pass over the domain list. The
// lanes of a warp holding pixels of one slot compare them with each of the slot's pairs and add the ballot counts.
__global__ void SuspectCount(Workspace ws)
{
	if (ws.cnt->nsuspect == 0) { return; }
	const uint32_t n = min(ws.cnt->ndom, ws.capDom);
	const int lane = threadIdx.x & 31;
	const uint32_t stride = gridDim.x * blockDim.x;
	// every lane of a warp runs the same iterations (the bound is rounded up to whole warps)
	const uint32_t nWarps = (n + 31u) & ~31u;
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nWarps; i += stride) {
		uint32_t s = 0, w = 0;
		bool poppable = false;
		if (i < n) {
			const uint32_t p = ws.dom[i];
			s = ws.frameSuspect[FastDivide(p, ws.g.divN)];
			if (s != 0u) {
				w = __ldg(ws.w1 + p);
				// every non-seed domain pixel is pushed and popped once; a seed only if it has a neighbour that is
				// not a seed (the reference's initial heap takes the labelled pixels next to an unlabelled one)
				poppable = !(__ldg(ws.code + p) & kSeed);
				if (!poppable) {
					const Pix q = Decompose(p, ws.g);
					for (int dy = -1; dy <= 1 && !poppable; ++dy) {
						const int yy = q.y + dy;
						if (yy < 0 || yy >= ws.g.H) { continue; }
						for (int dx = -1; dx <= 1 && !poppable; ++dx) {
							const int xx = q.x + dx;
							if ((dx == 0 && dy == 0) || xx < 0 || xx >= ws.g.W) { continue; }
							const uint32_t nb = p + static_cast<uint32_t>(dy * ws.g.W + dx);  // in the frame: no wrap
							poppable = !(__ldg(ws.code + nb) & kSeed);
						}
					}
				}
			}
		}
		unsigned pending = __ballot_sync(0xffffffffu, s != 0u);
		while (pending) {
			const uint32_t slot = __shfl_sync(0xffffffffu, s, __ffs(pending) - 1);
			const bool mine = s == slot;
			pending &= ~__ballot_sync(0xffffffffu, mine);
			const uint32_t k0 = ws.rankSlotOff[slot - 1u], k1 = ws.rankSlotOff[slot];
			for (uint32_t k = k0; k < k1; ++k) {
				const uint32_t idx = ws.rankOrder[k];
				const uint4 r = ws.suspect[idx];
				uint32_t lowB, lowA;
				PairLevels(ws, r, lowB, lowA);
				const uint32_t nb = __popc(__ballot_sync(0xffffffffu, mine && w >= lowB));
				const uint32_t na = __popc(__ballot_sync(0xffffffffu, mine && poppable && w > lowA));
				if (lane == 0) {
					if (nb) { atomicAdd(ws.rankCount + 2 * idx, nb); }
					if (na) { atomicAdd(ws.rankCount + 2 * idx + 1, na); }
				}
			}
		}
	}
}

// A frame that failed the rank test: flooded again per component with estimated frame-wide aging (reflood), or
// routed to the frame-wide flood.
__device__ __forceinline__ void FailRankTest(const Workspace& ws, int f, int reflood)
{
	if (!reflood) {
		RouteFrame(ws, f, kRouteRankFused);
		return;
	}
	if (atomicExch(ws.frameReflood + f, 1u) == 0u) { atomicAdd(&ws.cnt->nreflood, 1u); }
}

// Step 3: the rank test of every counted pair. reflood: frames that fail it are flooded again per component with
// estimated frame-wide aging (no basin fusion follows); else they are routed to the frame-wide flood.
__global__ void SuspectCheck(Workspace ws, int reflood)
{
	if (ws.cnt->nsuspect == 0) { return; }
	const uint32_t nrec = min(ws.cnt->nsuspect, ws.capSuspect);
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nrec; i += gridDim.x * blockDim.x) {
		const uint4 r = ws.suspect[i];
		if (ws.frameSuspect[r.x] == 0u) { continue; }  // no slot: the frame is routed already
		const long long bc = ws.rankCount[2 * i];
		const long long az = r.w == 0u ? 0ll : static_cast<long long>(ws.rankCount[2 * i + 1]) + 1;
		const long long lhs = (static_cast<long long>(r.y) - static_cast<long long>(r.z)) * 78125ll;
		if (!(lhs > (bc - az + 1) * 512ll)) { FailRankTest(ws, static_cast<int>(r.x), reflood); }
	}
}

// ---- Re-flood with estimated frame-wide aging -------------------------------------------------------------------
// A frame whose pairs fail the rank test may still be flooded per component: the test proves the labels of ANY
// per-component flood whose parent chains pass it, whatever aging that flood used. Its own flood used the local pop
// counter, which can order a contested pair differently from the frame-wide flood (the labels then genuinely
// differ); flooded again with each pop's push aging set to its estimated frame-wide position (the number of the
// frame's domain pixels with a higher W1, which the frame-wide flood pops first up to its aging term), the groups
// follow the frame-wide order, and the test, now with every chain element's own bound
//   min over e of (W1(e) * 78125 - B(parent(e)) * 512) > W1(z) * 78125 - (A_z - 1) * 512,
// B(p) = #{W1 >= W1(p) - delta}, proves it. The counts come from the frame's W1 values grouped by value bucket. A frame failing again
// (or beyond the slots or the value capacity) is flooded frame-wide.

// Step 1 (one CTA): slots for the frames marked by the rank test, in frame order; the others are routed.
__global__ void __launch_bounds__(kPlanThreads) RefloodPlan(Workspace ws)
{
	__shared__ uint32_t next;
	if (ws.cnt->nreflood == 0) { return; }
	if (threadIdx.x == 0) { next = 0; }
	if (threadIdx.x < kRefloodSlots * 8) { ws.rfInfo[threadIdx.x] = 0u; }
	__syncthreads();
	if (threadIdx.x == 0) {
		for (int f = 0; f < ws.g.B; ++f) {
			if (ws.frameReflood[f] == 0u) { continue; }
			if (next < kRefloodSlots && ws.frameRoute[f] == 0u && ws.frameDom[f] <= kRefloodCap) {
				ws.frameReflood[f] = next + 1u;
				ws.rfInfo[next * 8 + 2] = static_cast<uint32_t>(f) + 1u;
				++next;
			}
			else {
				ws.frameReflood[f] = 0u;
				RouteFrame(ws, f, kRouteRefloodSlots);
			}
		}
	}
}

// Pixel p (domain) of the chunk is popped by the frame-wide flood: a non-seed, or a seed with a non-seed neighbour
// (the reference's initial heap takes the labelled pixels next to an unlabelled one).
__device__ __forceinline__ bool Poppable(const Workspace& ws, uint32_t p)
{
	if (!(__ldg(ws.code + p) & kSeed)) { return true; }
	const Pix q = Decompose(p, ws.g);
	for (int dy = -1; dy <= 1; ++dy) {
		const int yy = q.y + dy;
		if (yy < 0 || yy >= ws.g.H) { continue; }
		for (int dx = -1; dx <= 1; ++dx) {
			const int xx = q.x + dx;
			if ((dx == 0 && dy == 0) || xx < 0 || xx >= ws.g.W) { continue; }
			const uint32_t nb = p + static_cast<uint32_t>(dy * ws.g.W + dx);
			if (!(__ldg(ws.code + nb) & kSeed)) { return true; }
		}
	}
	return false;
}

// Step 2: the W1 values of the slotted frames' domain pixels (and of their poppable pixels), read from the frames'
// code bytes, 16 pixels per thread with one atomic per warp and list; and the list of the slotted frames'
// multi-label groups, which the next steps walk instead of every group of the chunk.
__global__ void RefloodGather(Workspace ws)
{
	if (ws.cnt->nreflood == 0) { return; }
	const int lane = threadIdx.x & 31;
	const uint32_t N = static_cast<uint32_t>(ws.g.N);
	const uint32_t stride = gridDim.x * blockDim.x;  // whole warps
	// 16-pixel runs per frame, rounded up to whole warps: a warp never spans two slots, so it takes every branch below
	// as one
	const uint32_t per = ((N + 15u) / 16u + 31u) & ~31u;
	for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < kRefloodSlots * per; t += stride) {
		const uint32_t slot = t / per, q = t - slot * per;
		const uint32_t f1 = ws.rfInfo[slot * 8 + 2];  // frame + 1 (0: the slot is unused)
		if (f1 == 0u) { continue; }
		const uint32_t p0 = (f1 - 1u) * N;
		uint32_t dmask = 0, pmask = 0;
		for (uint32_t k = 0; k < 16u && q * 16u + k < N; ++k) {
			const uint32_t p = p0 + q * 16u + k;
			if (!(__ldg(ws.code + p) & kDomain)) { continue; }
			dmask |= 1u << k;
			if (Poppable(ws, p)) { pmask |= 1u << k; }
		}
		// both lists' positions from one scan (domain count in the low half, poppable count in the high half)
		const uint32_t c = static_cast<uint32_t>(__popc(dmask)) | (static_cast<uint32_t>(__popc(pmask)) << 16);
		uint32_t x = c;
		#pragma unroll
		for (int d = 1; d < 32; d <<= 1) {
			const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
			if (lane >= d) { x += y; }
		}
		uint32_t b0 = 0, b1 = 0;
		if (lane == 31) {
			b0 = (x & 0xffffu) ? atomicAdd(ws.rfInfo + slot * 8, x & 0xffffu) : 0u;
			b1 = (x >> 16) ? atomicAdd(ws.rfInfo + slot * 8 + 1, x >> 16) : 0u;
		}
		b0 = __shfl_sync(0xffffffffu, b0, 31) + ((x - c) & 0xffffu);
		b1 = __shfl_sync(0xffffffffu, b1, 31) + ((x - c) >> 16);
		uint32_t* vals = ws.rfVals + static_cast<size_t>(slot) * 2 * kRefloodCap;
		for (uint32_t b = dmask; b; b &= b - 1u) {
			const uint32_t k = static_cast<uint32_t>(__ffs(b) - 1), w = __ldg(ws.w1 + p0 + q * 16u + k);
			if (b0 < kRefloodCap) { vals[b0] = w; }
			++b0;
			if ((pmask >> k) & 1u) {
				if (b1 < kRefloodCap) { vals[kRefloodCap + b1] = w; }
				++b1;
			}
		}
	}
	const uint32_t nGroups = ws.cnt->nmulti;
	for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < nGroups; m += stride) {
		const uint32_t off = ws.gOff[m];
		if (ws.gOff[m + 1] == off || ws.frameReflood[FastDivide(ws.gPix[off], ws.g.divN)] == 0u) { continue; }
		ws.rfGroups[atomicAdd(&ws.cnt->nrfgroup, 1u)] = m;
	}
}

constexpr int kRfBucketThreads = 1024;
constexpr size_t kRfBucketSmem = kRefloodBuckets * sizeof(uint32_t);

// Step 3 (one CTA per slot and list): the values grouped by bucket (bucket = (value - lowest) >> shift, the shift the
// smallest that fits the value range in kRefloodBuckets buckets), bucket offsets by a counting pass in shared memory.
__global__ void __launch_bounds__(kRfBucketThreads) RefloodBucket(Workspace ws)
{
	extern __shared__ uint32_t hist[];  // [kRefloodBuckets]: counts, then cursors
	__shared__ uint32_t red[2][kRfBucketThreads / 32];
	__shared__ uint32_t carry;
	const uint32_t slot = blockIdx.x >> 1, a = blockIdx.x & 1u;
	if (ws.cnt->nreflood == 0 || ws.rfInfo[slot * 8 + 2] == 0u) { return; }
	const int tid = static_cast<int>(threadIdx.x), lane = tid & 31, warp = tid >> 5;
	const uint32_t* v = ws.rfVals + (static_cast<size_t>(slot) * 2 + a) * kRefloodCap;
	uint32_t* grp = ws.rfGrp + (static_cast<size_t>(slot) * 2 + a) * kRefloodCap;
	uint32_t* off = ws.rfOff + (static_cast<size_t>(slot) * 2 + a) * (kRefloodBuckets + 1);
	const uint32_t n = min(ws.rfInfo[slot * 8 + a], kRefloodCap);
	// value range
	uint32_t lo = 0xffffffffu, hi = 0u;
	for (uint32_t i = tid; i < n; i += kRfBucketThreads) {
		lo = min(lo, v[i]);
		hi = max(hi, v[i]);
	}
	#pragma unroll
	for (int d = 16; d > 0; d >>= 1) {
		lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, d));
		hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, d));
	}
	if (lane == 0) { red[0][warp] = lo; red[1][warp] = hi; }
	for (uint32_t b = tid; b < kRefloodBuckets; b += kRfBucketThreads) { hist[b] = 0u; }
	__syncthreads();
	lo = 0xffffffffu;
	hi = 0u;
	for (int w = 0; w < kRfBucketThreads / 32; ++w) {
		lo = min(lo, red[0][w]);
		hi = max(hi, red[1][w]);
	}
	if (n == 0) { lo = hi = 0u; }
	uint32_t shift = 0;
	while (shift < 32 && ((hi - lo) >> shift) >= kRefloodBuckets) { ++shift; }
	if (tid == 0) {
		ws.rfInfo[slot * 8 + 4 + 2 * a] = lo;
		ws.rfInfo[slot * 8 + 5 + 2 * a] = shift;
		carry = 0;
	}
	for (uint32_t i = tid; i < n; i += kRfBucketThreads) { atomicAdd(hist + ((v[i] - lo) >> shift), 1u); }
	__syncthreads();
	// exclusive scan of the bucket counts: each thread a run of buckets, then the runs before it
	constexpr uint32_t kRun = kRefloodBuckets / kRfBucketThreads;
	uint32_t sum = 0;
	for (uint32_t k = 0; k < kRun; ++k) { sum += hist[tid * kRun + k]; }
	uint32_t x = sum;
	#pragma unroll
	for (int d = 1; d < 32; d <<= 1) {
		const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
		if (lane >= d) { x += y; }
	}
	if (lane == 31) { red[0][warp] = x; }
	__syncthreads();
	if (warp == 0) {
		uint32_t w = red[0][lane];
		#pragma unroll
		for (int d = 1; d < 32; d <<= 1) {
			const uint32_t y = __shfl_up_sync(0xffffffffu, w, d);
			if (lane >= d) { w += y; }
		}
		red[1][lane] = w;  // inclusive over warps
	}
	__syncthreads();
	uint32_t run = (warp ? red[1][warp - 1] : 0u) + x - sum;
	for (uint32_t k = 0; k < kRun; ++k) {
		const uint32_t b = tid * kRun + k;
		const uint32_t c = hist[b];
		off[b] = run;
		hist[b] = run;  // cursor
		run += c;
	}
	if (tid == kRfBucketThreads - 1) { off[kRefloodBuckets] = run; }
	__syncthreads();
	for (uint32_t i = tid; i < n; i += kRfBucketThreads) {
		const uint32_t val = v[i];
		grp[atomicAdd(hist + ((val - lo) >> shift), 1u)] = val;
	}
}

// Values of list a of the slot that are >= x (strict: > x): the buckets above x's bucket, plus the members of its
// bucket counted one by one.
__device__ uint32_t CountAbove(const Workspace& ws, uint32_t slot, uint32_t a, uint32_t x, bool strict)
{
	const uint32_t n = min(ws.rfInfo[slot * 8 + a], kRefloodCap);
	const uint32_t lo = ws.rfInfo[slot * 8 + 4 + 2 * a], shift = ws.rfInfo[slot * 8 + 5 + 2 * a];
	if (n == 0) { return 0u; }
	if (x < lo) { return n; }
	const uint32_t b = shift >= 32 ? 0u : ((x - lo) >> shift);
	if (b >= kRefloodBuckets) { return 0u; }
	const uint32_t* off = ws.rfOff + (static_cast<size_t>(slot) * 2 + a) * (kRefloodBuckets + 1);
	const uint32_t* grp = ws.rfGrp + (static_cast<size_t>(slot) * 2 + a) * kRefloodCap;
	const uint32_t b0 = off[b], b1 = off[b + 1];
	uint32_t c = n - b1;
	for (uint32_t i = b0; i < b1; ++i) {
		const uint32_t y = grp[i];
		c += strict ? (y > x ? 1u : 0u) : (y >= x ? 1u : 0u);
	}
	return c;
}

__device__ __forceinline__ uint32_t FrameDelta(const Workspace& ws, int f)
{
	return static_cast<uint32_t>((static_cast<unsigned long long>(ws.frameDom[f]) * 65536ull) / 10000000ull) + 1u;
}

// Step 4: for every pixel of the slotted frames' listed groups (a warp per group): the estimated frame-wide pop position
// #{W1 > W1(p)} and its upper bound B(p) = #{W1 >= W1(p) - delta}.
__global__ void RefloodCounts(Workspace ws)
{
	if (ws.cnt->nreflood == 0) { return; }
	const uint32_t nList = ws.cnt->nrfgroup;
	const int lane = threadIdx.x & 31;
	const uint32_t warps = gridDim.x * (blockDim.x / 32);
	for (uint32_t g = (blockIdx.x * blockDim.x + threadIdx.x) / 32; g < nList; g += warps) {
		const uint32_t m = ws.rfGroups[g];
		const uint32_t off = ws.gOff[m], nPix = ws.gOff[m + 1] - off;
		if (nPix == 0) { continue; }
		const int f = Decompose(ws.gPix[off], ws.g).f;
		const uint32_t s = ws.frameReflood[f];
		if (s == 0u) { continue; }
		const uint32_t slot = s - 1u;
		const uint32_t delta = FrameDelta(ws, f);
		uint32_t* out = ws.rfPix + static_cast<size_t>(slot) * static_cast<size_t>(ws.g.N) * kRfWords;
		for (uint32_t i = lane; i < nPix; i += 32) {
			const uint32_t p = ws.gPix[off + i];
			const uint32_t w = __ldg(ws.w1 + p);
			const size_t local = static_cast<size_t>(p) - static_cast<size_t>(f) * static_cast<size_t>(ws.g.N);
			out[local * kRfWords] = CountAbove(ws, slot, 0, w, true);
			out[local * kRfWords + 1] = CountAbove(ws, slot, 0, w > delta ? w - delta : 0u, false);
		}
	}
}

constexpr int kRfWarps = 3;  // groups (warps) per CTA of the re-flood

struct RfBoxSmem {
	double key[kBoxHeap];
	uint32_t pix[kBoxHeap];
	long long v[kBoxCap];      // W1 * 78125 - B(pusher) * 512 (seeds: W1 * 78125)
	long long m[kBoxCap];      // minimum of v over the pusher's parent chain (seeds: none)
	uint32_t w1[kBoxCap];
	uint32_t lab[kBoxCap];
	uint32_t chain[kBoxCap];   // parent-chain minimum of W1 (the first test)
	uint32_t gest[kBoxCap];    // estimated frame-wide pop position
	uint32_t bnd[kBoxCap];     // its upper bound B
	uint8_t flag[kBoxCap];     // bit 0: domain; bit 1: a non-seed (flooded)
};

constexpr long long kNoM = 0x7fffffffffffffffll;

// Step 5 for a group larger than the shared-memory box (called by the whole warp): the same flood and test in global
// memory. Labels go to lab (the group's non-seed pixels restart unlabelled), chain minima to par (dead since the
// groups were scattered), element values v and their chain minima m to the slot's rfPix words 2-5; the heap spills to
// the group's global heap slice. Returns false when the frame must be flooded frame-wide.
__device__ bool RefloodGroupGlobal(const Workspace& ws, RfBoxSmem& sm, uint32_t m, uint32_t off, uint32_t nPix, int f,
                                   uint32_t slot)
{
	const int lane = threadIdx.x & 31;
	const Geometry& geo = ws.g;
	uint32_t* pix = ws.rfPix + static_cast<size_t>(slot) * static_cast<size_t>(geo.N) * kRfWords;
	const uint32_t frame0 = static_cast<uint32_t>(f) * static_cast<uint32_t>(geo.N);
	auto word = [&](uint32_t p) { return pix + static_cast<size_t>(p - frame0) * kRfWords; };
	auto getV = [&](uint32_t p, int k) {
		const uint32_t* q = word(p) + 2 + 2 * k;
		return static_cast<long long>((static_cast<unsigned long long>(q[1]) << 32) | q[0]);
	};
	auto setV = [&](uint32_t p, int k, long long x) {
		uint32_t* q = word(p) + 2 + 2 * k;
		q[0] = static_cast<uint32_t>(static_cast<unsigned long long>(x));
		q[1] = static_cast<uint32_t>(static_cast<unsigned long long>(x) >> 32);
	};
	for (uint32_t i = lane; i < nPix; i += 32) {
		const uint32_t p = ws.gPix[off + i];
		const bool seed = (__ldg(ws.code + p) & kSeed) != 0;
		if (!seed) { ws.lab[p] = 0u; }
		ws.par[p] = kNoChain;
		setV(p, 0, static_cast<long long>(__ldg(ws.w1 + p)) * 78125ll);  // a seed's value (no aging)
		setV(p, 1, kNoM);
	}
	__syncwarp();
	if (lane == 0) {
		uint32_t* seeds = ws.gSeed + ws.gSeedOff[m];
		const uint32_t nSeeds = ws.gSeedOff[m + 1] - ws.gSeedOff[m];
		SortSlice(seeds, nSeeds);
		Heap heap{sm.key, sm.pix, 0, 1, kBoxHeap, ws.heapKey + off, ws.heapPix + off};
		auto open = [&](uint32_t p, int y, int x) {
			for (int dy = -1; dy <= 1; ++dy) {
				const int yy = y + dy;
				if (yy < 0 || yy >= geo.H) { continue; }
				for (int dx = -1; dx <= 1; ++dx) {
					const int xx = x + dx;
					if ((dx == 0 && dy == 0) || xx < 0 || xx >= geo.W) { continue; }
					const uint32_t nb = p + static_cast<uint32_t>(dy * geo.W + dx);  // in the frame: no wrap
					if (!(__ldg(ws.code + nb) & kDomain) || ws.lab[nb] == 0u) { return true; }
				}
			}
			return false;
		};
		for (uint32_t k = 0; k < nSeeds; ++k) {
			const uint32_t sd = seeds[k];
			const Pix q = Decompose(sd, geo);
			if (open(sd, q.y, q.x)) { heap.Push(-(static_cast<double>(__ldg(ws.w1 + sd)) * kW1Unit), sd); }
		}
		while (heap.len > 0) {
			const uint32_t p = heap.Pop();
			const Pix q = Decompose(p, geo);
			const uint32_t L = ws.lab[p];
			const uint32_t* wp = word(p);
			// pushes at this pop age by the estimated frame-wide position of the pop
			const double age = __dmul_rn(static_cast<double>(wp[0]) + 1.0, kEps);
			const uint32_t chain = min(ws.par[p], __ldg(ws.w1 + p));
			const long long mch = min(getV(p, 1), getV(p, 0));
			const long long bpush = static_cast<long long>(wp[1]) * 512ll;
			for (int t = 0; t < 8; ++t) {
				const int dy = t < 3 ? -1 : (t < 5 ? 0 : 1);
				const int dx = t < 3 ? t - 1 : (t < 5 ? (t == 3 ? -1 : 1) : t - 6);
				const int yy = q.y + dy, xx = q.x + dx;
				if (yy < 0 || yy >= geo.H || xx < 0 || xx >= geo.W) { continue; }
				const uint32_t j = p + static_cast<uint32_t>(dy * geo.W + dx);
				if (!(__ldg(ws.code + j) & kDomain) || ws.lab[j] != 0u) { continue; }
				const uint32_t wj = __ldg(ws.w1 + j);
				heap.Push(__dadd_rn(-(static_cast<double>(wj) * kW1Unit), age), j);
				ws.lab[j] = L;
				ws.par[j] = chain;
				setV(j, 1, mch);
				setV(j, 0, static_cast<long long>(wj) * 78125ll - bpush);
			}
		}
	}
	__syncwarp();
	// the per-element test at every boundary pair of a flooded pixel that fails the first test
	const uint32_t T = ws.frameDom[f];
	const uint32_t delta = FrameDelta(ws, f);
	bool exact = true;
	for (uint32_t i = lane; i < nPix && exact; i += 32) {
		const uint32_t p = ws.gPix[off + i];
		if (__ldg(ws.code + p) & kSeed) { continue; }
		const uint32_t L = ws.lab[p], chain = ws.par[p];
		if (L == 0u) { continue; }
		const long long mi = getV(p, 1);
		const Pix q = Decompose(p, geo);
		for (int dy = -1; dy <= 1 && exact; ++dy) {
			if (q.y + dy < 0 || q.y + dy >= geo.H) { continue; }
			for (int dx = -1; dx <= 1 && exact; ++dx) {
				if ((dx == 0 && dy == 0) || q.x + dx < 0 || q.x + dx >= geo.W) { continue; }
				const uint32_t j = p + static_cast<uint32_t>(dy * geo.W + dx);
				if (!(__ldg(ws.code + j) & kDomain) || ws.lab[j] == L) { continue; }
				const uint32_t wj = __ldg(ws.w1 + j);
				if (PairExact(chain, wj, T)) { continue; }
				long long az = 0;
				if (ws.par[j] != kNoChain) {  // z pushed: its pusher is one of its neighbours, none above zmax
					uint32_t zmax = 0;
					const int zy = q.y + dy, zx = q.x + dx;
					for (int ey = -1; ey <= 1; ++ey) {
						if (zy + ey < 0 || zy + ey >= geo.H) { continue; }
						for (int ex = -1; ex <= 1; ++ex) {
							if ((ex == 0 && ey == 0) || zx + ex < 0 || zx + ex >= geo.W) { continue; }
							const uint32_t e = j + static_cast<uint32_t>(ey * geo.W + ex);
							if (__ldg(ws.code + e) & kDomain) { zmax = max(zmax, __ldg(ws.w1 + e)); }
						}
					}
					const unsigned long long x = static_cast<unsigned long long>(zmax) + delta;
					az = (x < 0xffffffffull ? static_cast<long long>(CountAbove(ws, slot, 1, static_cast<uint32_t>(x), true)) : 0ll) + 1;
				}
				if (!(mi > static_cast<long long>(wj) * 78125ll - (az - 1) * 512ll)) { exact = false; }
			}
		}
	}
	return __all_sync(0xffffffffu, exact) != 0;
}

// Step 5: warp per group of the slotted frames, box staged in shared memory (a larger group: RefloodGroupGlobal):
// the flood with push aging (estimated position + 1) * 1e-7, then the per-element test at every boundary pair that
// fails the first test; a failing frame is routed to the frame-wide flood.
__global__ void __launch_bounds__(kRfWarps * 32) RefloodBox(Workspace ws)
{
	__shared__ RfBoxSmem boxes[kRfWarps];
	if (ws.cnt->nreflood == 0) { return; }
	RfBoxSmem& sm = boxes[threadIdx.x / 32];
	const int lane = threadIdx.x & 31;
	const Geometry& geo = ws.g;
	const uint32_t nList = ws.cnt->nrfgroup;
	for (uint32_t g = blockIdx.x * kRfWarps + threadIdx.x / 32; g < nList; g += gridDim.x * kRfWarps) {
		const uint32_t m = ws.rfGroups[g];
		const uint32_t off = ws.gOff[m], nPix = ws.gOff[m + 1] - off;
		if (nPix == 0) { continue; }
		const int f = Decompose(ws.gPix[off], geo).f;  // every lane reads the group's first pixel
		const uint32_t s = ws.frameReflood[f];
		if (s == 0u || ws.frameRoute[f] != 0u) { continue; }
		const uint32_t slot = s - 1u;
		int x0 = geo.W, y0 = geo.H, x1 = -1, y1 = -1;
		for (uint32_t i = lane; i < nPix; i += 32) {
			const Pix q = Decompose(ws.gPix[off + i], geo);
			x0 = min(x0, q.x); x1 = max(x1, q.x); y0 = min(y0, q.y); y1 = max(y1, q.y);
		}
		#pragma unroll
		for (int d = 16; d > 0; d >>= 1) {
			x0 = min(x0, __shfl_xor_sync(0xffffffffu, x0, d));
			y0 = min(y0, __shfl_xor_sync(0xffffffffu, y0, d));
			x1 = max(x1, __shfl_xor_sync(0xffffffffu, x1, d));
			y1 = max(y1, __shfl_xor_sync(0xffffffffu, y1, d));
		}
		const int bx0 = max(x0 - 1, 0), by0 = max(y0 - 1, 0);
		const int bw = min(x1 + 1, geo.W - 1) - bx0 + 1, bh = min(y1 + 1, geo.H - 1) - by0 + 1;
		if (bw * bh > kBoxCap) {
			if (!RefloodGroupGlobal(ws, sm, m, off, nPix, f, slot) && lane == 0) { RouteFrame(ws, f, kRouteRefloodTest); }
			continue;
		}
		const uint32_t base = static_cast<uint32_t>(f) * static_cast<uint32_t>(geo.N) + static_cast<uint32_t>(by0 * geo.W + bx0);
		const uint32_t* pix = ws.rfPix + static_cast<size_t>(slot) * static_cast<size_t>(geo.N) * kRfWords;
		const uint32_t local0 = static_cast<uint32_t>(by0 * geo.W + bx0);
		for (int i = lane; i < bw * bh; i += 32) {
			const int r = i / bw, c = i - r * bw;
			const uint32_t p = base + static_cast<uint32_t>(r * geo.W + c);
			const uint8_t code = __ldg(ws.code + p);
			const bool dom = (code & kDomain) != 0, seed = (code & kSeed) != 0;
			const uint32_t w = dom ? __ldg(ws.w1 + p) : 0u;
			sm.w1[i] = w;
			sm.lab[i] = dom && seed ? ws.lab[p] : 0u;
			sm.chain[i] = kNoChain;
			sm.flag[i] = static_cast<uint8_t>((dom ? 1u : 0u) | (dom && !seed ? 2u : 0u));
			const size_t local = static_cast<size_t>(local0) + static_cast<size_t>(r) * geo.W + c;
			sm.gest[i] = dom ? pix[local * kRfWords] : 0u;
			sm.bnd[i] = dom ? pix[local * kRfWords + 1] : 0u;
			sm.v[i] = static_cast<long long>(w) * 78125ll;  // a seed's value (no aging); pushed pixels overwrite it
			sm.m[i] = kNoM;
		}
		__syncwarp();
		if (lane == 0) {
			uint32_t* seeds = ws.gSeed + ws.gSeedOff[m];
			const uint32_t nSeeds = ws.gSeedOff[m + 1] - ws.gSeedOff[m];
			SortSlice(seeds, nSeeds);
			Heap heap{sm.key, sm.pix, 0, 1, kBoxHeap, ws.heapKey + off, ws.heapPix + off};
			auto at = [&](int y, int x) { return (y - by0) * bw + (x - bx0); };
			for (uint32_t k = 0; k < nSeeds; ++k) {
				const uint32_t sd = seeds[k];
				const Pix q = Decompose(sd, geo);
				bool open = false;
				for (int dy = -1; dy <= 1 && !open; ++dy) {
					const int yy = q.y + dy;
					if (yy < 0 || yy >= geo.H) { continue; }
					for (int dx = -1; dx <= 1 && !open; ++dx) {
						const int xx = q.x + dx;
						if ((dx == 0 && dy == 0) || xx < 0 || xx >= geo.W) { continue; }
						const int j = at(yy, xx);
						if (!(sm.flag[j] & 1u) || sm.lab[j] == 0) { open = true; }
					}
				}
				if (open) { heap.Push(-(static_cast<double>(sm.w1[at(q.y, q.x)]) * kW1Unit), sd); }
			}
			while (heap.len > 0) {
				const uint32_t p = heap.Pop();
				const Pix q = Decompose(p, geo);
				const int ip = at(q.y, q.x);
				const uint32_t L = sm.lab[ip];
				// pushes at this pop age by the estimated frame-wide position of the pop
				const double age = __dmul_rn(static_cast<double>(sm.gest[ip]) + 1.0, kEps);
				const uint32_t chain = min(sm.chain[ip], sm.w1[ip]);
				const long long mch = min(sm.m[ip], sm.v[ip]);
				const long long bpush = static_cast<long long>(sm.bnd[ip]) * 512ll;
				for (int t = 0; t < 8; ++t) {
					const int dy = t < 3 ? -1 : (t < 5 ? 0 : 1);
					const int dx = t < 3 ? t - 1 : (t < 5 ? (t == 3 ? -1 : 1) : t - 6);
					const int yy = q.y + dy, xx = q.x + dx;
					if (yy < 0 || yy >= geo.H || xx < 0 || xx >= geo.W) { continue; }
					const int j = at(yy, xx);
					if (!(sm.flag[j] & 1u) || sm.lab[j] != 0) { continue; }
					const double k = __dadd_rn(-(static_cast<double>(sm.w1[j]) * kW1Unit), age);
					heap.Push(k, p + static_cast<uint32_t>(dy * geo.W + dx));
					sm.lab[j] = L;
					sm.chain[j] = chain;
					sm.m[j] = mch;
					sm.v[j] = static_cast<long long>(sm.w1[j]) * 78125ll - bpush;
				}
			}
		}
		__syncwarp();
		const uint32_t T = ws.frameDom[f];
		const uint32_t delta = FrameDelta(ws, f);
		bool exact = true;
		for (int i = lane; i < bw * bh; i += 32) {
			if (!(sm.flag[i] & 2u) || sm.lab[i] == 0) { continue; }
			const int r = i / bw, c = i - r * bw;
			ws.lab[base + static_cast<uint32_t>(r * geo.W + c)] = sm.lab[i];
			const uint32_t L = sm.lab[i], chain = sm.chain[i];
			const long long mi = sm.m[i];
			for (int dy = -1; dy <= 1; ++dy) {
				if (r + dy < 0 || r + dy >= bh) { continue; }
				for (int dx = -1; dx <= 1; ++dx) {
					if ((dx == 0 && dy == 0) || c + dx < 0 || c + dx >= bw) { continue; }
					const int j = i + dy * bw + dx;
					if (!(sm.flag[j] & 1u) || sm.lab[j] == L || PairExact(chain, sm.w1[j], T)) { continue; }
					long long az = 0;
					if (sm.chain[j] != kNoChain) {  // z pushed: its pusher is one of its neighbours, none above zmax
						uint32_t zmax = 0;
						const int zr = r + dy, zc = c + dx;
						for (int ey = -1; ey <= 1; ++ey) {
							if (zr + ey < 0 || zr + ey >= bh) { continue; }
							for (int ex = -1; ex <= 1; ++ex) {
								if ((ex == 0 && ey == 0) || zc + ex < 0 || zc + ex >= bw) { continue; }
								zmax = max(zmax, sm.w1[j + ey * bw + ex]);
							}
						}
						const unsigned long long x = static_cast<unsigned long long>(zmax) + delta;
						az = (x < 0xffffffffull ? static_cast<long long>(CountAbove(ws, slot, 1, static_cast<uint32_t>(x), true)) : 0ll) + 1;
					}
					if (!(mi > static_cast<long long>(sm.w1[j]) * 78125ll - (az - 1) * 512ll)) { exact = false; }
				}
			}
		}
		if (__any_sync(0xffffffffu, !exact) && lane == 0) { RouteFrame(ws, f, kRouteRefloodTest); }
		__syncwarp();
	}
}

// Exact integer sums per region (ComputeStatistics, Segmentation2D.cpp:144-175).
// Consecutive domain-list entries of one warp that belong to the same region are summed with shuffles first, so
// there is one set of atomics per run instead of per pixel (integer sums: the order does not matter).
__global__ void RegionStats(Workspace ws)
{
	const uint32_t n = min(ws.cnt->ndom, ws.capDom);
	const Geometry& geo = ws.g;
	PTB_WARP_LOOP(k, n)
	{
		uint32_t r = 0xffffffffu;
		unsigned long long v = 0, vx = 0, vy = 0;
		if (k < n) {
			const uint32_t p = ws.dom[k];
			const uint32_t L = ws.lab[p];
			if (L != 0) {
				r = L - 1;
				const Pix q = Decompose(p, geo);
				v = static_cast<unsigned long long>(ws.w1[p]);
				vx = v * static_cast<unsigned long long>(q.x);
				vy = v * static_cast<unsigned long long>(q.y);
			}
		}
		bool head;
		const uint32_t cnt = RunSum<uint32_t>(r, r != 0xffffffffu ? 1u : 0u, head);
		v = RunSum<unsigned long long>(r, v, head);
		vx = RunSum<unsigned long long>(r, vx, head);
		vy = RunSum<unsigned long long>(r, vy, head);
		if (head && r != 0xffffffffu) {
			atomicAdd(ws.regCount + r, cnt);
			atomicAdd(ws.regSumV + r, v);
			atomicAdd(ws.regSumVJ + r, vx);
			atomicAdd(ws.regSumVI + r, vy);
		}
	}
}

__global__ void CandidateFlags(Workspace ws)
{
	const uint32_t n = ws.cnt->nregion;
	for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
		ws.regCand[r] = static_cast<double>(ws.regCount[r]) > kVolumeMin ? 1u : 0u;  // FilterData, :88-141
	}
}

// Per frame: candidate base, kept count (capacity truncation in label order, Fitting.cpp:44-58) and output base.
__global__ void FrameCandidates(Workspace ws, uint32_t maxPoints)
{
	const int B = ws.g.B;
	for (int f = blockIdx.x * blockDim.x + threadIdx.x; f <= B; f += gridDim.x * blockDim.x) {
		const uint32_t rb = ws.rowcnt[static_cast<long long>(f) * ws.g.H];
		ws.frameRegBase[f] = rb;
		ws.frameCandBase[f] = ws.regCand[rb];
	}
}

__global__ void FrameKeep(Workspace ws, uint32_t maxPoints)
{
	const int B = ws.g.B;
	for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < B; f += gridDim.x * blockDim.x) {
		const uint32_t c = ws.frameCandBase[f + 1] - ws.frameCandBase[f];
		ws.frameKeep[f] = min(c, maxPoints);
		if (c > maxPoints) { atomicExch(&ws.cnt->truncated, 1u); }
	}
}

__global__ void CandidateEmit(Workspace ws, uint32_t maxPoints)
{
	const uint32_t n = ws.cnt->nregion;
	for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
		if (!(static_cast<double>(ws.regCount[r]) > kVolumeMin)) { continue; }
		const int f = ws.regFrame[r];
		const uint32_t k = ws.regCand[r] - ws.frameCandBase[f];
		if (k >= maxPoints) { continue; }
		const uint32_t slot = ws.frameOutBase[f] + k;
		if (slot >= ws.capRows) { atomicExch(&ws.cnt->overflow, 1u); continue; }
		ws.candRegion[slot] = r;
		ws.candFrame[slot] = static_cast<uint32_t>(f);
	}
}

}  // namespace

// Runs the whole segmentation of a chunk after detection. `strict` selects frame-wide floods.
bool LaunchSegment(const Workspace& ws, double ratio, int strict, uint32_t maxPoints, cudaStream_t st)
{
	const Geometry& g = ws.g;
	bool ok = true;
	CclInit<<<kGrid, kThreads, 0, st>>>(ws);
	CclUnion<<<kGrid, kThreads, 0, st>>>(ws);
	CompEnumerate<<<kGrid, kThreads, 0, st>>>(ws);
	CompCount<<<kGrid, kThreads, 0, st>>>(ws);
	SeedParent<<<kGrid, kThreads, 0, st>>>(ws);
	RowCount<<<kGrid, kThreads, 0, st>>>(ws);
	CountLaunch(6);
	ok = ok && PTB_LAUNCHED();
	const uint32_t rows = static_cast<uint32_t>(g.B) * static_cast<uint32_t>(g.H);
	ok = ok && ExclusiveScan(ws.rowcnt, nullptr, rows, rows, ws.scanBlock, &ws.cnt->nregion, st);
	SeedLabel<<<kGrid, kThreads, 0, st>>>(ws);
	CountLaunch();
	ok = ok && PTB_LAUNCHED();
	// mode 0: per-component floods with both exactness tests; 2: with the first test only; 1: frame-wide floods
	const int rank = strict == 0 ? 1 : 0;
	strict = strict == 1 ? 1 : 0;
	const uint32_t groupsStrict = strict ? static_cast<uint32_t>(g.B) : 0u;
	if (strict) {
		PTB_CUDA(cudaMemsetAsync(ws.gOff, 0, sizeof(uint32_t) * (g.B + 1), st));
		PTB_CUDA(cudaMemsetAsync(ws.gSeedOff, 0, sizeof(uint32_t) * (g.B + 1), st));
		PTB_CUDA(cudaMemsetAsync(ws.gRegOff, 0, sizeof(uint32_t) * (g.B + 1), st));
		PTB_CUDA(cudaMemsetAsync(ws.gCurPix, 0, sizeof(uint32_t) * (g.B + 1), st));
		PTB_CUDA(cudaMemsetAsync(ws.gCurSeed, 0, sizeof(uint32_t) * (g.B + 1), st));
		PTB_CUDA(cudaMemsetAsync(ws.gCurReg, 0, sizeof(uint32_t) * (g.B + 1), st));
		GroupSizesStrict<<<kGrid, kThreads, 0, st>>>(ws);
		CountLaunch();
		ok = ok && PTB_LAUNCHED();
		ok = ok && ExclusiveScan(ws.gOff, nullptr, groupsStrict, groupsStrict, ws.scanBlock, nullptr, st);
		ok = ok && ExclusiveScan(ws.gSeedOff, nullptr, groupsStrict, groupsStrict, ws.scanBlock, nullptr, st);
		ok = ok && ExclusiveScan(ws.gRegOff, nullptr, groupsStrict, groupsStrict, ws.scanBlock, nullptr, st);
	}
	else {
		GroupEnumerate<<<kGrid, kThreads, 0, st>>>(ws);
		CountLaunch();
		ok = ok && PTB_LAUNCHED();
		ok = ok && ExclusiveScan(ws.gOff, &ws.cnt->nmulti, 0, ws.capComp, ws.scanBlock, nullptr, st);
		ok = ok && ExclusiveScan(ws.gSeedOff, &ws.cnt->nmulti, 0, ws.capComp, ws.scanBlock, nullptr, st);
		ok = ok && ExclusiveScan(ws.gRegOff, &ws.cnt->nmulti, 0, ws.capComp, ws.scanBlock, nullptr, st);
	}
	GroupScatter<<<kGrid, kThreads, 0, st>>>(ws, strict ? 1 : 0);
	if (strict) {  // frame-wide groups: one thread per group, small CTAs so that many SMs share the frames
		GroupFlood<<<kGrid * 2, kFloodThreads, 0, st>>>(ws, groupsStrict, 0);
	}
	else {  // one warp per group, staged in shared memory
		GroupFloodBox<<<kGrid, kBoxWarps * 32, 0, st>>>(ws, rank);
	}
	CountLaunch(2);
	ok = ok && PTB_LAUNCHED();
	const bool fuse = static_cast<int>(ratio) > 0;  // WatershedIntelligent, Segmentation2D.cpp:77-85
	if (fuse) {
		GroupFuse<<<kGrid * 2, kFloodThreads, 0, st>>>(ws, groupsStrict, ratio, 0);
		CountLaunch();
		ok = ok && PTB_LAUNCHED();
	}
	if (!strict) {
		// boundary pairs that failed the first exactness test: the rank test of their frames (each kernel returns at
		// once when no pair failed)
		if (rank) {
			SuspectPlan<<<1, kPlanThreads, 0, st>>>(ws);
			SuspectCount<<<kGrid, kThreads, 0, st>>>(ws);
			// frames failing the rank test: flooded again with estimated frame-wide aging (not after a basin fusion,
			// which used the first flood's labels)
			SuspectCheck<<<64, kThreads, 0, st>>>(ws, fuse ? 0 : 1);
			RefloodPlan<<<1, kPlanThreads, 0, st>>>(ws);
			RefloodGather<<<kGrid, kThreads, 0, st>>>(ws);
			static const bool bucketSmem = PTB_CUDA(cudaFuncSetAttribute(RefloodBucket, cudaFuncAttributeMaxDynamicSharedMemorySize,
			                                                             static_cast<int>(kRfBucketSmem)));
			ok = ok && bucketSmem;
			RefloodBucket<<<kRefloodSlots * 2, kRfBucketThreads, kRfBucketSmem, st>>>(ws);
			RefloodCounts<<<kGrid, kThreads, 0, st>>>(ws);
			RefloodBox<<<kGrid, kRfWarps * 32, 0, st>>>(ws);
			CountLaunch(8);
			ok = ok && PTB_LAUNCHED();
		}
		// frames whose per-component floods failed the exactness tests: flooded again as one unit with the frame-global
		// pop counter (each kernel returns at once when no frame was routed)
		const uint32_t frames = static_cast<uint32_t>(g.B);
		RedoOffsets<<<1, kRedoThreads, 0, st>>>(ws);
		GroupScatter<<<kGrid, kThreads, 0, st>>>(ws, 2);
		GroupFlood<<<kGrid * 2, kFloodThreads, 0, st>>>(ws, frames, 1);
		CountLaunch(3);
		if (fuse) {
			GroupFuse<<<kGrid * 2, kFloodThreads, 0, st>>>(ws, frames, ratio, 1);
			CountLaunch();
		}
		ok = ok && PTB_LAUNCHED();
	}
	RegionStats<<<kGrid, kThreads, 0, st>>>(ws);
	CandidateFlags<<<kGrid, kThreads, 0, st>>>(ws);
	CountLaunch(2);
	ok = ok && PTB_LAUNCHED();
	ok = ok && ExclusiveScan(ws.regCand, &ws.cnt->nregion, 0, ws.capRegion, ws.scanBlock, &ws.cnt->ncand, st);
	FrameCandidates<<<(g.B + 256) / 256, 256, 0, st>>>(ws, maxPoints);
	FrameKeep<<<(g.B + 255) / 256, 256, 0, st>>>(ws, maxPoints);
	CountLaunch(2);
	ok = ok && PTB_LAUNCHED();
	PTB_CUDA(cudaMemcpyAsync(ws.frameOutBase, ws.frameKeep, sizeof(uint32_t) * g.B, cudaMemcpyDeviceToDevice, st));
	ok = ok && ExclusiveScan(ws.frameOutBase, nullptr, static_cast<uint32_t>(g.B), static_cast<uint32_t>(g.B), ws.scanBlock,
	                         &ws.cnt->nfit, st);
	CandidateEmit<<<kGrid, kThreads, 0, st>>>(ws, maxPoints);
	CountLaunch();
	ok = ok && PTB_LAUNCHED();
	return ok;
}

}  // namespace ptb
