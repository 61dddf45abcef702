// Streaming detection front end: the exact fixed-point B3 a trous wavelet, the strict threshold and the local maxima,
// with each warp sweeping one strip of the frame down a block of rows. Same results as DetectKernel (detect.cu),
// which covers frames too small for a strip; the arithmetic, the units and the reference citations are the ones
// documented there (lib/localization/ATrous.cpp:23-80, Segmentation2D.cpp:50-74 and :294-333).
//
// A lane owns 4 consecutive columns, a warp 128: the strip's 112 output columns (lanes 2-29) and 8 halo columns on
// each side. The iteration that receives input row r computes four stages, each from rows finished in earlier
// iterations so that the four are independent of one another:
//   1. H1(r), the horizontal level-1 taps of the input row;
//   2. V1(r - 3), the vertical level-1 taps of the H1 rows r - 5 .. r - 1;
//   3. W1(r - 8) = V1 * 256 - V2, where V2 = H2 taps of the vertical level-2 taps of the V1 rows r - 12 .. r - 4
//      (both level-2 directions are linear in the integers, so taking the vertical taps first gives the same V2);
//   4. the threshold, the 3 x 3 maximum and the outputs of row r - 10 (W1 rows r - 11 .. r - 9).
// Horizontal neighbours come from the adjacent lanes by shuffles, vertical ones from per-warp row rings in shared
// memory in which each lane reads and writes only its own word (no bank conflicts, no barrier). Input rows arrive
// kAhead rows ahead by asynchronous copies when the frame width is a multiple of 4 (8-byte lane loads).
// Borders: every pass evaluates its output at the clamped coordinate, as the reference's offsetTest() does: input
// rows and columns are read clamped, V1 rows outside the frame repeat the nearest row, the vertical level-2 taps
// outside the frame repeat the nearest column, and W1 is 0 outside the frame.
#include "pt_common.cuh"
#include "async_copy.cuh"

namespace ptb {

long long ThresholdFixed(double thr);

namespace {

constexpr int kStripOut = 112;  // output columns per warp
constexpr int kRowsOut = 256;   // output rows per warp
constexpr int kSWarps = 2;      // strips per CTA
constexpr int kListBuf = 128;   // domain and seed list entries staged per warp before one atomic reserves their range
constexpr int kAhead = 8;       // input rows in flight per warp

struct StreamSmem {
	uint2 in[kAhead][32];  // input rows in flight (4 columns per lane), ring by iteration
	uint4 h1[8][32];       // H1 rows, ring by row & 7
	uint4 v1[16][32];      // V1 rows, ring by row & 15 (rows -4 .. -1 and H .. H + 3 repeat the nearest row)
	uint4 w1[4][32];       // W1 rows (0 outside the frame), ring by row & 3
	uint32_t w1l[4][32], w1r[4][32];  // W1 of the column left of the lane's first and right of its last
	uint32_t dom[kListBuf];
	uint32_t seed[kListBuf];
};
constexpr size_t kStreamSmem = kSWarps * sizeof(StreamSmem);

__device__ __forceinline__ uint32_t Tap(uint32_t m2, uint32_t m1, uint32_t c, uint32_t p1, uint32_t p2)
{
	return 6u * c + 4u * (m1 + p1) + (m2 + p2);
}

__device__ __forceinline__ int Clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ uint32_t Elem(const uint4& v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w)); }

__device__ __forceinline__ uint4 Tap4(const uint4& a, const uint4& b, const uint4& c, const uint4& d, const uint4& e)
{
	return make_uint4(Tap(a.x, b.x, c.x, d.x, e.x), Tap(a.y, b.y, c.y, d.y, e.y), Tap(a.z, b.z, c.z, d.z, e.z),
	                  Tap(a.w, b.w, c.w, d.w, e.w));
}

__device__ __forceinline__ uint32_t Max3(uint32_t a, uint32_t b, uint32_t c) { return max(a, max(b, c)); }

// Bits 0-3 of m to the low bits of bytes 0-3.
__device__ __forceinline__ uint32_t Spread4(uint32_t m) { return (m * 0x00204081u) & 0x01010101u; }

// Replaces the elements of v at columns outside the frame by the element at the nearest column inside it (held by
// lane hold >> 2, element hold & 3). Called by all 32 lanes of an edge strip.
__device__ __forceinline__ void RepeatLeft(uint4& v, int cx, int hold)
{
	const uint32_t b = __shfl_sync(0xffffffffu, Elem(v, hold & 3), hold >> 2);
	if (cx < 0) { v.x = b; }
	if (cx + 1 < 0) { v.y = b; }
	if (cx + 2 < 0) { v.z = b; }
	if (cx + 3 < 0) { v.w = b; }
}

__device__ __forceinline__ void RepeatRight(uint4& v, int cx, int W, int hold)
{
	const uint32_t b = __shfl_sync(0xffffffffu, Elem(v, hold & 3), hold >> 2);
	if (cx > W - 1) { v.x = b; }
	if (cx + 1 > W - 1) { v.y = b; }
	if (cx + 2 > W - 1) { v.z = b; }
	if (cx + 3 > W - 1) { v.w = b; }
}

// Adds this row's entries of one list (pixel g0 + k for bit k of each lane's mask; `before` entries of lower lanes,
// `total` in the warp) to the warp's stage in shared memory, first moving a stage that would overflow to the global
// list with one atomic. n is the stage's fill, the same in every lane. Called by all 32 lanes.
__device__ __forceinline__ void Stage(uint32_t mask, uint32_t g0, uint32_t before, uint32_t total, uint32_t* buf,
                                      uint32_t& n, uint32_t* counter, uint32_t* list, uint32_t cap, uint32_t* overflow)
{
	if (total == 0) { return; }
	const int lane = threadIdx.x & 31;
	if (n + total > kListBuf) {
		__syncwarp();  // the other lanes' entries are visible
		uint32_t base = 0;
		if (lane == 0) { base = atomicAdd(counter, n); }
		base = __shfl_sync(0xffffffffu, base, 0);
		for (uint32_t i = lane; i < n; i += 32) {
			if (base + i < cap) { list[base + i] = buf[i]; }
			else { atomicExch(overflow, 1u); }
		}
		__syncwarp();  // every entry is read before the stage is refilled
		n = 0;
	}
	uint32_t pos = n + before;
	for (uint32_t b = mask; b; b &= b - 1u) { buf[pos++] = g0 + static_cast<uint32_t>(__ffs(b) - 1); }
	n += total;
}

__device__ __forceinline__ void Drain(const uint32_t* buf, uint32_t n, uint32_t* counter, uint32_t* list, uint32_t cap,
                                      uint32_t* overflow)
{
	const int lane = threadIdx.x & 31;
	__syncwarp();
	uint32_t base = 0;
	if (lane == 0 && n) { base = atomicAdd(counter, n); }
	base = __shfl_sync(0xffffffffu, base, 0);
	for (uint32_t i = lane; i < n; i += 32) {
		if (base + i < cap) { list[base + i] = buf[i]; }
		else { atomicExch(overflow, 1u); }
	}
}

// kVec: the frame width is a multiple of 4 and the frames are 8-byte aligned, so each lane's 4 input columns are one
// aligned 8-byte word (lanes outside the frame read the nearest word inside and take the edge pixel by a shuffle)
// and rows arrive by asynchronous copies kAhead rows ahead. Otherwise each lane reads its 4 clamped columns directly.
template <bool kVec>
__global__ void __launch_bounds__(kSWarps * 32) DetectStream(const uint16_t* __restrict__ img, Workspace ws, long long thrFixed)
{
	extern __shared__ __align__(16) unsigned char streamRaw[];
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	StreamSmem& sm = reinterpret_cast<StreamSmem*>(streamRaw)[warp];
	const int H = ws.g.H, W = ws.g.W;
	const int X0 = (blockIdx.x * kSWarps + warp) * kStripOut;
	if (X0 >= W) { return; }  // the whole warp
	const int Y0 = blockIdx.y * kRowsOut, Y1 = min(Y0 + kRowsOut, H), f = blockIdx.z;
	const uint16_t* frame = img + static_cast<long long>(f) * ws.g.N;
	const int cx = X0 - 8 + 4 * lane;  // this lane's first column
	const bool leftEdge = X0 - 8 < 0, rightEdge = X0 + 120 > W;
	// the lanes and elements holding columns 0 and W - 1
	const int lOff = 8 - X0, rOff = W - 1 - (X0 - 8);
	const uint32_t thr = thrFixed <= 0 ? 0u : (thrFixed >= 0xffffffffll ? 0xffffffffu : static_cast<uint32_t>(thrFixed));
	const bool outLane = lane >= 2 && lane < 30;
	const int rFirst = Y0 - 7, rIn = Y1 + 7;  // input rows rFirst .. rIn - 1 are read
	const int raLo = max(0, Y0 - 5), raHi = min(H - 1, Y1 + 4);  // V1 rows needed
	const int rbLo = max(0, Y0 - 1), rbHi = min(H - 1, Y1);      // W1 rows needed
	const int lx = Clampi(cx, 0, W - 4);  // kVec: the aligned word this lane reads
	if (kVec) {
		#pragma unroll
		for (int j = 0; j < kAhead; ++j) {
			const int rr = rFirst + j;
			if (rr < rIn) { CpAsync8(&sm.in[j][lane], frame + static_cast<long long>(Clampi(rr, 0, H - 1)) * W + lx); }
			CpAsyncCommit();
		}
	}
	uint32_t nDomStage = 0, nSeedStage = 0, cntDom = 0, cntSeed = 0;  // the same in every lane
	for (int r = rFirst; r < Y1 + 10; ++r) {
		// 1. input row r and its H1
		if (r < rIn) {
			uint32_t in0, in1, in2, in3;
			const int slot = (r - rFirst) & (kAhead - 1);
			if (kVec) {
				CpAsyncWait<kAhead - 1>();  // the group of row r (one group per row, committed in row order)
				const uint2 q = sm.in[slot][lane];
				in0 = q.x & 0xffffu; in1 = q.x >> 16; in2 = q.y & 0xffffu; in3 = q.y >> 16;
				if (leftEdge) {  // lanes left of column 0 take pixel 0 (lane 2, element 0)
					const uint32_t t = __shfl_sync(0xffffffffu, in0, 2);
					if (cx < 0) { in0 = t; in1 = t; in2 = t; in3 = t; }
				}
				if (rightEdge) {  // lanes right of column W - 1 take pixel W - 1 (element 3 of the lane reading W - 4)
					const uint32_t t = __shfl_sync(0xffffffffu, in3, (W - 4 - (X0 - 8)) >> 2);
					if (cx >= W) { in0 = t; in1 = t; in2 = t; in3 = t; }
				}
			}
			else {
				const uint16_t* row = frame + static_cast<long long>(Clampi(r, 0, H - 1)) * W;
				in0 = __ldg(row + Clampi(cx, 0, W - 1));
				in1 = __ldg(row + Clampi(cx + 1, 0, W - 1));
				in2 = __ldg(row + Clampi(cx + 2, 0, W - 1));
				in3 = __ldg(row + Clampi(cx + 3, 0, W - 1));
			}
			const uint32_t pl = __shfl_up_sync(0xffffffffu, in2 | (in3 << 16), 1);    // columns cx - 2, cx - 1
			const uint32_t pr = __shfl_down_sync(0xffffffffu, in0 | (in1 << 16), 1);  // columns cx + 4, cx + 5
			const uint32_t l0 = pl & 0xffffu, l1 = pl >> 16, r0 = pr & 0xffffu, r1v = pr >> 16;
			sm.h1[r & 7][lane] = make_uint4(Tap(l0, l1, in0, in1, in2), Tap(l1, in0, in1, in2, in3), Tap(in0, in1, in2, in3, r0),
			                                Tap(in1, in2, in3, r0, r1v));
			if (kVec) {  // the slot is free again (its row went into the shuffles): row r + kAhead into it
				const int rr = r + kAhead;
				if (rr < rIn) { CpAsync8(&sm.in[slot][lane], frame + static_cast<long long>(Clampi(rr, 0, H - 1)) * W + lx); }
				CpAsyncCommit();
			}
		}
		// 2. V1 of row r - 3
		const int ra = r - 3;
		if (ra >= raLo && ra <= raHi) {
			const uint4 v = Tap4(sm.h1[(ra - 2) & 7][lane], sm.h1[(ra - 1) & 7][lane], sm.h1[ra & 7][lane],
			                     sm.h1[(ra + 1) & 7][lane], sm.h1[(ra + 2) & 7][lane]);
			sm.v1[ra & 15][lane] = v;
			// rows outside the frame: the nearest row's (the level-2 vertical taps read them at clamped rows)
			if (ra == 0) {
				#pragma unroll
				for (int k = 1; k <= 4; ++k) { sm.v1[(-k) & 15][lane] = v; }
			}
			if (ra == H - 1) {
				#pragma unroll
				for (int k = 1; k <= 4; ++k) { sm.v1[(H - 1 + k) & 15][lane] = v; }
			}
		}
		// 3. W1 of row r - 8
		const int rb = r - 8;
		if (rb >= rbLo && rb <= rbHi) {
			const uint4 c = sm.v1[rb & 15][lane];
			uint4 t = Tap4(sm.v1[(rb - 4) & 15][lane], sm.v1[(rb - 2) & 15][lane], c, sm.v1[(rb + 2) & 15][lane],
			               sm.v1[(rb + 4) & 15][lane]);
			if (leftEdge) { RepeatLeft(t, cx, lOff); }
			if (rightEdge) { RepeatRight(t, cx, W, rOff); }
			uint32_t u[12];
			u[0] = __shfl_up_sync(0xffffffffu, t.x, 1);
			u[1] = __shfl_up_sync(0xffffffffu, t.y, 1);
			u[2] = __shfl_up_sync(0xffffffffu, t.z, 1);
			u[3] = __shfl_up_sync(0xffffffffu, t.w, 1);
			u[4] = t.x; u[5] = t.y; u[6] = t.z; u[7] = t.w;
			u[8] = __shfl_down_sync(0xffffffffu, t.x, 1);
			u[9] = __shfl_down_sync(0xffffffffu, t.y, 1);
			u[10] = __shfl_down_sync(0xffffffffu, t.z, 1);
			u[11] = __shfl_down_sync(0xffffffffu, t.w, 1);
			const uint32_t v2x = Tap(u[0], u[2], u[4], u[6], u[8]), v2y = Tap(u[1], u[3], u[5], u[7], u[9]);
			const uint32_t v2z = Tap(u[2], u[4], u[6], u[8], u[10]), v2w = Tap(u[3], u[5], u[7], u[9], u[11]);
			uint4 w;
			w.x = (cx >= 0 && cx < W) ? max(c.x << 8, v2x) - v2x : 0u;
			w.y = (cx + 1 >= 0 && cx + 1 < W) ? max(c.y << 8, v2y) - v2y : 0u;
			w.z = (cx + 2 >= 0 && cx + 2 < W) ? max(c.z << 8, v2z) - v2z : 0u;
			w.w = (cx + 3 >= 0 && cx + 3 < W) ? max(c.w << 8, v2w) - v2w : 0u;
			sm.w1[rb & 3][lane] = w;
			sm.w1l[rb & 3][lane] = __shfl_up_sync(0xffffffffu, w.w, 1);
			sm.w1r[rb & 3][lane] = __shfl_down_sync(0xffffffffu, w.x, 1);
		}
		// 4. threshold, 3 x 3 maximum and outputs of row r - 10
		const int y = r - 10;
		if (y >= Y0 && y < Y1) {
			uint32_t a[3][6];
			#pragma unroll
			for (int dy = -1; dy <= 1; ++dy) {
				const int yy = y + dy;
				if (yy < 0 || yy >= H) {
					#pragma unroll
					for (int j = 0; j < 6; ++j) { a[dy + 1][j] = 0u; }
				}
				else {
					const uint4 q = sm.w1[yy & 3][lane];
					a[dy + 1][0] = sm.w1l[yy & 3][lane];
					a[dy + 1][1] = q.x; a[dy + 1][2] = q.y; a[dy + 1][3] = q.z; a[dy + 1][4] = q.w;
					a[dy + 1][5] = sm.w1r[yy & 3][lane];
				}
			}
			uint32_t cm[6];
			#pragma unroll
			for (int j = 0; j < 6; ++j) { cm[j] = Max3(a[0][j], a[1][j], a[2][j]); }
			uint32_t dm = 0, smk = 0;
			#pragma unroll
			for (int k = 0; k < 4; ++k) {
				const uint32_t v = a[1][k + 1];
				const bool dom = outLane && cx + k < W && v > thr;
				dm |= static_cast<uint32_t>(dom) << k;
				smk |= static_cast<uint32_t>(dom && v >= Max3(cm[k], cm[k + 1], cm[k + 2])) << k;
			}
			const uint32_t g0 = static_cast<uint32_t>(f) * static_cast<uint32_t>(ws.g.N) + static_cast<uint32_t>(y) * W + cx;
			if (outLane && cx < W) {
				const uint32_t bytes = Spread4(dm) * kDomain | Spread4(smk) * kSeed;
				if (cx + 4 <= W && (g0 & 3) == 0) { *reinterpret_cast<uint32_t*>(ws.code + g0) = bytes; }
				else {
					for (int k = 0; k < 4 && cx + k < W; ++k) { ws.code[g0 + k] = static_cast<uint8_t>(bytes >> (8 * k)); }
				}
				#pragma unroll
				for (int k = 0; k < 4; ++k) {
					if ((dm >> k) & 1u) { ws.w1[g0 + k] = a[1][k + 1]; }
				}
			}
			// both lists' counts in one scan (domain in the low half, seeds in the high half; each at most 112)
			const uint32_t c = static_cast<uint32_t>(__popc(dm)) | (static_cast<uint32_t>(__popc(smk)) << 16);
			uint32_t x = c;
			#pragma unroll
			for (int d = 1; d < 32; d <<= 1) {
				const uint32_t z = __shfl_up_sync(0xffffffffu, x, d);
				if (lane >= d) { x += z; }
			}
			const uint32_t tot = __shfl_sync(0xffffffffu, x, 31), ex = x - c;
			cntDom += tot & 0xffffu;
			cntSeed += tot >> 16;
			Stage(dm, g0, ex & 0xffffu, tot & 0xffffu, sm.dom, nDomStage, &ws.cnt->ndom, ws.dom, ws.capDom, &ws.cnt->overflow);
			Stage(smk, g0, ex >> 16, tot >> 16, sm.seed, nSeedStage, &ws.cnt->nseed, ws.seeds, ws.capSeed, &ws.cnt->overflow);
		}
	}
	Drain(sm.dom, nDomStage, &ws.cnt->ndom, ws.dom, ws.capDom, &ws.cnt->overflow);
	Drain(sm.seed, nSeedStage, &ws.cnt->nseed, ws.seeds, ws.capSeed, &ws.cnt->overflow);
	// per-frame counts (the watershed's exactness bound)
	if (lane == 0) {
		if (cntDom) { atomicAdd(ws.frameDom + f, cntDom); }
		if (cntSeed) { atomicAdd(ws.frameSeeds + f, cntSeed); }
	}
}

template <bool kVec> bool LaunchStream(const Workspace& ws, double thr, cudaStream_t st)
{
	static const bool configured = PTB_CUDA(cudaFuncSetAttribute(DetectStream<kVec>, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                                                             static_cast<int>(kStreamSmem)));
	if (!configured) { return false; }
	const int strips = (ws.g.W + kStripOut - 1) / kStripOut;
	const dim3 grid((strips + kSWarps - 1) / kSWarps, (ws.g.H + kRowsOut - 1) / kRowsOut, ws.g.B);
	DetectStream<kVec><<<grid, kSWarps * 32, kStreamSmem, st>>>(ws.img, ws, ThresholdFixed(thr));
	CountLaunch();
	return PTB_LAUNCHED();
}

}  // namespace

// Frames at least one strip wide and 16 rows high go through the streaming kernel (16 rows keep the V1 ring's
// repeated border rows apart from the rows in use).
bool StreamDetectFits(int H, int W) { return W >= kStripOut && H >= 16; }

bool LaunchDetectStream(const Workspace& ws, double thr, cudaStream_t st)
{
	const bool vec = (ws.g.W & 3) == 0 && (reinterpret_cast<uintptr_t>(ws.img) & 7) == 0;
	return vec ? LaunchStream<true>(ws, thr, st) : LaunchStream<false>(ws, thr, st);
}

}  // namespace ptb
