// Streaming detection front end: the exact fixed-point B3 a trous wavelet, the strict threshold and the local maxima,
// with each warp sweeping one strip of the frame down a block of rows. Same results as DetectKernel (detect.cu),
// which covers frames too small for a strip; the arithmetic, the units and the reference citations are the ones
// documented there (lib/localization/ATrous.cpp:23-80, Segmentation2D.cpp:50-74 and :294-333).
//
// A lane owns 4 consecutive columns, a warp 128: the strip's 112 output columns (lanes 2-29) and 8 halo columns on
// each side. Row r of the input yields, in the same iteration, the horizontal level-1 taps H1(r), V1(r - 2) (vertical
// taps of the H1 rows r - 4 .. r), the level-2 horizontal taps H2(r - 2) of V1 at +-2, +-4 columns, V2 and
// W1 = V1 * 256 - V2 of row r - 6 (vertical level-2 taps of the H2 rows r - 10 .. r - 2) and the threshold and 3 x 3
// maximum of output row r - 7. Horizontal neighbours come from the adjacent lanes by shuffles, vertical ones from
// per-warp row rings in shared memory in which each lane reads and writes only its own 16-byte word (no bank
// conflicts, no barrier). Borders: every pass evaluates its output at the clamped coordinate, as the reference's
// offsetTest() does: input rows and columns are loaded clamped, V1 outside the frame takes the value of the nearest
// column in the frame, H2 rows outside the frame that of the nearest row, and W1 is 0 outside the frame.
#include "pt_common.cuh"

namespace ptb {

long long ThresholdFixed(double thr);

namespace {

constexpr int kStripOut = 112;  // output columns per warp
constexpr int kRowsOut = 128;   // output rows per warp
constexpr int kSWarps = 4;      // strips per CTA
constexpr int kListBuf = 256;   // domain and seed list entries staged per warp before one atomic reserves their range

struct StreamSmem {
	uint4 h1[8][32];   // H1 rows, ring by row & 7
	uint4 v1[8][32];   // V1 rows, ring by row & 7
	uint4 h2[16][32];  // H2 rows, ring by row & 15
	uint4 w1[4][32];   // W1 rows (0 outside the frame), ring by row & 3
	uint32_t w1l[4][32], w1r[4][32];  // W1 of the column left of the lane's first and right of its last
	uint32_t dom[kListBuf];
	uint32_t seed[kListBuf];
	uint32_t ndom, nseed;
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

// Appends the entries of the lanes' 4-bit masks (pixel g0 + k for bit k) to a list staged in shared memory; a full
// stage is first moved to the global list with one atomic. Called by all 32 lanes.
__device__ __forceinline__ void Append(uint32_t mask, uint32_t g0, uint32_t* buf, uint32_t& nbuf, uint32_t* counter,
                                       uint32_t* list, uint32_t cap, uint32_t* overflow)
{
	const int lane = threadIdx.x & 31;
	const uint32_t c = __popc(mask);
	uint32_t x = c;
	#pragma unroll
	for (int d = 1; d < 32; d <<= 1) {
		const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
		if (lane >= d) { x += y; }
	}
	const uint32_t total = __shfl_sync(0xffffffffu, x, 31);
	if (total == 0) { return; }
	uint32_t n = nbuf;  // read by every lane (written only by lane 0, behind the __syncwarp below)
	if (n + total > kListBuf) {
		uint32_t base = 0;
		if (lane == 0) { base = atomicAdd(counter, n); }
		base = __shfl_sync(0xffffffffu, base, 0);
		for (uint32_t i = lane; i < n; i += 32) {
			if (base + i < cap) { list[base + i] = buf[i]; }
			else { atomicExch(overflow, 1u); }
		}
		n = 0;
		__syncwarp();
	}
	uint32_t pos = n + x - c;
	for (uint32_t b = mask; b; b &= b - 1u) { buf[pos++] = g0 + static_cast<uint32_t>(__ffs(b) - 1); }
	__syncwarp();
	if (lane == 0) { nbuf = n + total; }
	__syncwarp();
}

__device__ __forceinline__ void Flush(const uint32_t* buf, uint32_t& nbuf, uint32_t* counter, uint32_t* list, uint32_t cap,
                                      uint32_t* overflow)
{
	const int lane = threadIdx.x & 31;
	const uint32_t n = nbuf;
	uint32_t base = 0;
	if (lane == 0 && n) { base = atomicAdd(counter, n); }
	base = __shfl_sync(0xffffffffu, base, 0);
	for (uint32_t i = lane; i < n; i += 32) {
		if (base + i < cap) { list[base + i] = buf[i]; }
		else { atomicExch(overflow, 1u); }
	}
	__syncwarp();
}

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
	const bool vec = !leftEdge && !rightEdge && (W & 3) == 0 && (reinterpret_cast<uintptr_t>(frame) & 7) == 0;
	// the lanes and elements holding columns 0 and W - 1 (replication of V1 outside the frame)
	const int lOff = 8 - X0, rOff = W - 1 - (X0 - 8);
	const uint32_t thr = thrFixed <= 0 ? 0u : (thrFixed >= 0xffffffffll ? 0xffffffffu : static_cast<uint32_t>(thrFixed));
	const bool outLane = lane >= 2 && lane < 30;
	if (lane == 0) {
		sm.ndom = 0;
		sm.nseed = 0;
	}
	__syncwarp();
	uint32_t cntDom = 0, cntSeed = 0;
	for (int r = Y0 - 7; r < Y1 + 7; ++r) {
		// input row r (clamped) and H1 of its 4 columns
		const uint16_t* row = frame + static_cast<long long>(Clampi(r, 0, H - 1)) * W;
		uint32_t in0, in1, in2, in3;
		if (vec) {
			const uint2 q = __ldg(reinterpret_cast<const uint2*>(row + cx));
			in0 = q.x & 0xffffu; in1 = q.x >> 16; in2 = q.y & 0xffffu; in3 = q.y >> 16;
		}
		else {
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
		// V1 and H2 of row r - 2 (rows in the frame that the W1 rows of this block need)
		const int ra = r - 2;
		if (ra >= 0 && ra < H && ra >= Y0 - 5 && ra <= Y1 + 4) {
			uint4 v = Tap4(sm.h1[(ra - 2) & 7][lane], sm.h1[(ra - 1) & 7][lane], sm.h1[ra & 7][lane], sm.h1[(ra + 1) & 7][lane],
			               sm.h1[(ra + 2) & 7][lane]);
			if (leftEdge) {
				const uint32_t b = __shfl_sync(0xffffffffu, Elem(v, lOff & 3), lOff >> 2);
				if (cx < 0) { v.x = b; }
				if (cx + 1 < 0) { v.y = b; }
				if (cx + 2 < 0) { v.z = b; }
				if (cx + 3 < 0) { v.w = b; }
			}
			if (rightEdge) {
				const uint32_t b = __shfl_sync(0xffffffffu, Elem(v, rOff & 3), rOff >> 2);
				if (cx > W - 1) { v.x = b; }
				if (cx + 1 > W - 1) { v.y = b; }
				if (cx + 2 > W - 1) { v.z = b; }
				if (cx + 3 > W - 1) { v.w = b; }
			}
			sm.v1[ra & 7][lane] = v;
			uint32_t u[12];
			u[0] = __shfl_up_sync(0xffffffffu, v.x, 1);
			u[1] = __shfl_up_sync(0xffffffffu, v.y, 1);
			u[2] = __shfl_up_sync(0xffffffffu, v.z, 1);
			u[3] = __shfl_up_sync(0xffffffffu, v.w, 1);
			u[4] = v.x; u[5] = v.y; u[6] = v.z; u[7] = v.w;
			u[8] = __shfl_down_sync(0xffffffffu, v.x, 1);
			u[9] = __shfl_down_sync(0xffffffffu, v.y, 1);
			u[10] = __shfl_down_sync(0xffffffffu, v.z, 1);
			u[11] = __shfl_down_sync(0xffffffffu, v.w, 1);
			const uint4 h2 = make_uint4(Tap(u[0], u[2], u[4], u[6], u[8]), Tap(u[1], u[3], u[5], u[7], u[9]),
			                            Tap(u[2], u[4], u[6], u[8], u[10]), Tap(u[3], u[5], u[7], u[9], u[11]));
			sm.h2[ra & 15][lane] = h2;
			// H2 rows outside the frame: the nearest row's (the level-2 vertical taps read them at clamped rows)
			if (ra == 0) {
				#pragma unroll
				for (int k = 1; k <= 4; ++k) { sm.h2[(-k) & 15][lane] = h2; }
			}
			if (ra == H - 1) {
				#pragma unroll
				for (int k = 1; k <= 4; ++k) { sm.h2[(H - 1 + k) & 15][lane] = h2; }
			}
		}
		// V2 and W1 of row r - 6
		const int rb = r - 6;
		if (rb >= 0 && rb < H && rb >= Y0 - 1 && rb <= Y1) {
			const uint4 v2 = Tap4(sm.h2[(rb - 4) & 15][lane], sm.h2[(rb - 2) & 15][lane], sm.h2[rb & 15][lane],
			                      sm.h2[(rb + 2) & 15][lane], sm.h2[(rb + 4) & 15][lane]);
			const uint4 v1 = sm.v1[rb & 7][lane];
			uint4 w;
			w.x = (cx >= 0 && cx < W) ? max(v1.x << 8, v2.x) - v2.x : 0u;
			w.y = (cx + 1 >= 0 && cx + 1 < W) ? max(v1.y << 8, v2.y) - v2.y : 0u;
			w.z = (cx + 2 >= 0 && cx + 2 < W) ? max(v1.z << 8, v2.z) - v2.z : 0u;
			w.w = (cx + 3 >= 0 && cx + 3 < W) ? max(v1.w << 8, v2.w) - v2.w : 0u;
			sm.w1[rb & 3][lane] = w;
			sm.w1l[rb & 3][lane] = __shfl_up_sync(0xffffffffu, w.w, 1);
			sm.w1r[rb & 3][lane] = __shfl_down_sync(0xffffffffu, w.x, 1);
		}
		// threshold, 3 x 3 maximum and outputs of row r - 7
		const int y = r - 7;
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
				const bool in = outLane && cx + k < W;
				const bool dom = in && v > thr;
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
				for (uint32_t b = dm; b; b &= b - 1u) {
					const int k = __ffs(b) - 1;
					ws.w1[g0 + k] = a[1][k + 1];
				}
			}
			cntDom += __popc(dm);
			cntSeed += __popc(smk);
			Append(dm, g0, sm.dom, sm.ndom, &ws.cnt->ndom, ws.dom, ws.capDom, &ws.cnt->overflow);
			Append(smk, g0, sm.seed, sm.nseed, &ws.cnt->nseed, ws.seeds, ws.capSeed, &ws.cnt->overflow);
		}
	}
	Flush(sm.dom, sm.ndom, &ws.cnt->ndom, ws.dom, ws.capDom, &ws.cnt->overflow);
	Flush(sm.seed, sm.nseed, &ws.cnt->nseed, ws.seeds, ws.capSeed, &ws.cnt->overflow);
	// per-frame counts (the watershed's exactness bound); a list beyond its capacity marks the chunk for a redo
	#pragma unroll
	for (int d = 16; d > 0; d >>= 1) {
		cntDom += __shfl_xor_sync(0xffffffffu, cntDom, d);
		cntSeed += __shfl_xor_sync(0xffffffffu, cntSeed, d);
	}
	if (lane == 0) {
		if (cntDom) { atomicAdd(ws.frameDom + f, cntDom); }
		if (cntSeed) { atomicAdd(ws.frameSeeds + f, cntSeed); }
	}
}

}  // namespace

// Frames at least one strip wide and one row block high go through the streaming kernel.
bool StreamDetectFits(int H, int W) { return W >= kStripOut && H >= 16; }

bool LaunchDetectStream(const Workspace& ws, double thr, cudaStream_t st)
{
	static const bool configured = PTB_CUDA(cudaFuncSetAttribute(DetectStream, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                                                             static_cast<int>(kStreamSmem)));
	if (!configured) { return false; }
	const int strips = (ws.g.W + kStripOut - 1) / kStripOut;
	const dim3 grid((strips + kSWarps - 1) / kSWarps, (ws.g.H + kRowsOut - 1) / kRowsOut, ws.g.B);
	DetectStream<<<grid, kSWarps * 32, kStreamSmem, st>>>(ws.img, ws, ThresholdFixed(thr));
	CountLaunch();
	return PTB_LAUNCHED();
}

}  // namespace ptb
