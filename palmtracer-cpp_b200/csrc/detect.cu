// Detection front end: exact fixed-point B3 a trous wavelet, strict threshold and local maxima, one tile per CTA.
//
// Reference: lib/localization/ATrous.cpp:23-80 (FP64 separable passes with clamped borders), thresholding in
// lib/localization/Segmentation2D.cpp:50-74 and seeds in :294-333.
//
// Why integers: the B3 taps are 1/16 * {1, 4, 6, 4, 1} and the input is uint16, so every FP64 value the reference
// computes for planes 0-2 is an exact dyadic rational (V1 in units of 2^-8, V2 and W1 in units of 2^-16). Integer
// arithmetic in those units reproduces the reference bit for bit, independent of summation order or FMA contraction:
//   T1 = sum h' * in          (units 1/16,  < 2^20, uint32)
//   V1 = sum h' * T1          (units 1/256, < 2^24)
//   T2 = sum h' * V1 at +-2,4 (units 2^-12, < 2^28)
//   V2 = sum h' * T2          (units 2^-16, < 2^32, fits uint32)
//   W1 = V1 * 256 - V2        (units 2^-16, |W1| < 2^32; kept as max(W1, 0) in uint32)
// with h' = {1, 4, 6, 4, 1}. Each pass evaluates its output at the CLAMPED coordinate, exactly like the reference's
// offsetTest() clamping of every neighbour access, so border tiles need no special case. The strict threshold
// W1 > thr is evaluated as W1_fixed > floor(thr * 2^16), which is the same test for an integer W1_fixed.
//
// Layout: a 128 x 28 output tile per CTA of 8 warps (the Wavelett planes: every stage loops rows over warps and
// columns over lanes; shared buffers are reused across stages, input -> V1, T1 -> T2).
#include <cuda.h>  // CUtensorMap and the tensor-map encoder's types (the encoder is fetched from the driver at run time)

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "pt_common.cuh"

namespace ptb {

namespace {

constexpr int TX = 128, TY = 28;          // output tile (28 rows: 44 KB of shared memory, 5 CTAs per SM)
constexpr int HIN = 7;                    // input halo: W1 on the tile +-1 ring needs V2 +-1, V1 +-5, input +-7
constexpr int IW = TX + 2 * HIN, IH = TY + 2 * HIN;
constexpr int V1W = TX + 10, V1H = TY + 10;
constexpr int RW = TX + 2, RH = TY + 2;  // ring region (tile +-1)
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

struct TileSmem {
	union {
		uint16_t in[IH][IW];
		uint32_t v1[V1H][V1W];
	} a;
	union {
		uint32_t t1[IH][V1W];
		uint32_t t2[V1H][RW];
	} b;
	uint32_t v2[RH][RW];
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Fills s.a.v1 (V1 on tile +-5) and s.v2 (V2 on tile +-1), all at clamped coordinates.
__device__ void WaveletTile(TileSmem& s, const uint16_t* __restrict__ frame, int H, int W, int x0, int y0)
{
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	for (int r = warp; r < IH; r += kWarps) {
		const uint16_t* row = frame + static_cast<long long>(clampi(y0 - HIN + r, 0, H - 1)) * W;
		for (int c = lane; c < IW; c += 32) { s.a.in[r][c] = __ldg(row + clampi(x0 - HIN + c, 0, W - 1)); }
	}
	__syncthreads();
	// row pass 1 (step 1): all input rows, V1 columns
	for (int r = warp; r < IH; r += kWarps) {
		const uint16_t* row = s.a.in[r];
		for (int c = lane; c < V1W; c += 32) {
			const int cx = clampi(x0 - 5 + c, 0, W - 1) - (x0 - HIN);
			s.b.t1[r][c] = 6u * row[cx] + 4u * (static_cast<uint32_t>(row[cx - 1]) + row[cx + 1]) +
			               (static_cast<uint32_t>(row[cx - 2]) + row[cx + 2]);
		}
	}
	__syncthreads();
	// column pass 1 (step 1): V1 on tile +-5 (the input buffer is no longer read and is reused)
	for (int r = warp; r < V1H; r += kWarps) {
		const int cy = clampi(y0 - 5 + r, 0, H - 1) - (y0 - HIN);
		for (int c = lane; c < V1W; c += 32) {
			s.a.v1[r][c] = 6u * s.b.t1[cy][c] + 4u * (s.b.t1[cy - 1][c] + s.b.t1[cy + 1][c]) + (s.b.t1[cy - 2][c] + s.b.t1[cy + 2][c]);
		}
	}
	__syncthreads();
	// row pass 2 (step 2): V1 rows, ring columns (overwrites T1)
	for (int r = warp; r < V1H; r += kWarps) {
		const uint32_t* row = s.a.v1[r];
		for (int c = lane; c < RW; c += 32) {
			const int cx = clampi(x0 - 1 + c, 0, W - 1) - (x0 - 5);
			s.b.t2[r][c] = 6u * row[cx] + 4u * (row[cx - 2] + row[cx + 2]) + (row[cx - 4] + row[cx + 4]);
		}
	}
	__syncthreads();
	// column pass 2 (step 2): V2 on tile +-1
	for (int r = warp; r < RH; r += kWarps) {
		const int cy = clampi(y0 - 1 + r, 0, H - 1) - (y0 - 5);
		for (int c = lane; c < RW; c += 32) {
			s.v2[r][c] = 6u * s.b.t2[cy][c] + 4u * (s.b.t2[cy - 2][c] + s.b.t2[cy + 2][c]) + (s.b.t2[cy - 4][c] + s.b.t2[cy + 4][c]);
		}
	}
	__syncthreads();
}

// W1 at ring position (r, c): V1 * 256 - V2 in 2^-16 units.
__device__ __forceinline__ long long W1At(const TileSmem& s, int r, int c)
{
	return static_cast<long long>(s.a.v1[r + 4][c + 4]) * 256 - static_cast<long long>(s.v2[r][c]);
}

// ---- Detection kernel ------------------------------------------------------------------------------------------
// The input box of a tile is first staged in shared memory: by one TMA bulk tensor copy where the frames' width is a
// multiple of 8 (StageTma, then StageFixBorders on border tiles; measured 400 against 362 GB/s of input for the
// per-thread loads on the 2000-frame 1024 x 1024 benchmark), else by per-thread loads; then five register-blocked passes over one
// 128 x 28 tile (44 KB of shared memory, so 5 CTAs per SM; 128 x 32 took 49.7 KB, 4 CTAs per SM, and measured 2 %
// slower for 2 % less halo work). Borders: every intermediate array is kept edge-replicated
// (an entry whose coordinate lies outside the frame holds the value of the nearest in-frame entry), which is what
// the reference's clamping of every neighbour access amounts to, so no pass clamps an index:
//   A  C1 = vertical level-1 taps of the input, one lane per column and run of 13 rows sliding down the clamped
//      input rows;                       tile rows [-5, 33), cols [-7, 145)
//   B  V1 = horizontal level-1 taps of C1, 4 columns per task from 2 vector loads, each C1 row outside the frame
//      read at the nearest in-frame row (columns outside the frame are then replicated);
//                                        tile rows [-5, 33), cols [-5, 139)
//   C  C2 = vertical level-2 taps (rows +-2, +-4) of V1, one lane per column and 12-row run;   rows [-1, 29)
//   D  W1 = V1 * 256 - V2 on the ring (tile +-1), V2 = horizontal level-2 taps of C2, 4 columns per task, stored
//      in place of V1 as max(W1, 0) (W1 < 2^32; a non-positive W1 can neither be in the domain nor dominate a
//      domain pixel) and 0 outside the frame (the reference skips neighbours outside the frame);
//   E  threshold and 3 x 3 maximum for 4 pixels per task; code bytes, W1 of domain pixels (uint32), and the domain
//      and seed lists with one atomic per block and list.
// In passes B, D and E consecutive lanes read and write consecutive 16-byte words, so no two lanes of a quarter
// warp share a shared-memory bank.
constexpr int kP1 = 152;  // C1 pitch (tile col = index - 7); C2 (pitch kPV, tile col = index - 5) reuses its space
constexpr int kPV = 144;  // V1 pitch (tile col = index - 5, tile row = index - 5); W1 ring in place
constexpr int kRows1 = TY + 10;  // C1 and V1 rows
constexpr int kRows2 = TY + 2;   // C2 rows and ring rows (tile row = index - 1)
constexpr int kV1Off = (kRows1 * kP1 + 31) / 32 * 32;  // V1 (and the staged input) start 128-byte aligned
constexpr int kDetectWords = kV1Off + kRows1 * kPV;
constexpr int kDetectBytes = kDetectWords * 4 + 128;  // + the alignment slack of the dynamic area's base
constexpr int kInRows = TY + 14, kInW = 160;  // staged input tile (uint16): rows y0-7.., columns x0-8..
static_assert(kRows2 * kPV <= kRows1 * kP1, "C2 must fit in the C1 space");
static_assert(kInRows * kInW * 2 <= kRows1 * kPV * 4, "the staged input must fit in the V1 space");
static_assert(kInW % 8 == 0 && kInW <= 256 && kInRows <= 256, "TMA box: 16-byte rows, at most 256 per dimension");
static_assert(kP1 + 1 <= kInW, "C1 columns read staged columns 1 .. kP1");
static_assert(kRows2 <= 36, "pass C covers C2 rows in three runs of 12");
constexpr int kRunA = 13, kRunsA = (kRows1 + kRunA - 1) / kRunA;  // pass A: rows per run, runs per column
constexpr int kTasksD = (TX + 2 + 3) / 4;                          // pass D: 4-column tasks per ring row
constexpr int kTasksE = (TY * (TX / 4) + kThreads - 1) / kThreads;  // pass E: 4-pixel tasks per thread
static_assert(kPV % 4 == 0 && kP1 % 4 == 0, "16-byte rows");
static_assert(4 * (kPV / 4 - 1) + 7 < kP1, "pass B reads C1 columns 4m .. 4m + 7");
static_assert(4 * (kTasksD - 1) + 11 < kPV && 4 * (kTasksD - 1) + 7 < kPV, "pass D stays inside C2 and V1 rows");
static_assert(4 * 31 + 11 < kPV, "pass E reads ring columns 4m .. 4m + 7");
static_assert(TX / 4 == 32 && kTasksE * 4 <= 32, "pass E: one warp per tile row, 4 bits per task in a mask");

// ---- Input staging by the tensor memory accelerator (TMA) -------------------------------------------------------
// The stack is described to the TMA as a 3-D uint16 tensor [frames][H][W] (x fastest; needs W a multiple of 8 and a
// 16-byte aligned base, so that the row and frame strides are multiples of 16 bytes). One elected thread copies the
// whole kInRows x kInW input box of a tile (rows y0-7.., columns x0-8..; x0 - 8 is a multiple of 8, so the box's x
// coordinate is 16-byte aligned) with one cp.async.bulk.tensor that completes on an mbarrier; the box may start above
// or left of the frame and reach past it, and the TMA fills those entries with zeros. The reference clamps every
// neighbour access into the frame instead, so border tiles then replicate the nearest in-frame column and row into
// the zero-filled entries (StageFixBorders).
constexpr long long kTmaWaitCycles = 4000000000ll;  // about 2 s at the B200's 1965 MHz: a bound, never reached

__device__ __forceinline__ uint32_t SmemAddr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// Waits until the mbarrier's phase `parity` has completed, at most kTmaWaitCycles; false when the bound ran out.
__device__ __forceinline__ bool MbarWaitBounded(uint32_t bar, uint32_t parity)
{
#if defined(__CUDA_ARCH__)
	const long long t0 = clock64();
	while (true) {
		uint32_t done;
		asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
		             : "=r"(done) : "r"(bar), "r"(parity) : "memory");
		if (done) { return true; }
		if (clock64() - t0 > kTmaWaitCycles) { return false; }
	}
#else
	(void)bar; (void)parity;
	return true;
#endif
}

// Copies the tile's input box into `in` (kInRows x kInW uint16, 128-byte aligned) through the TMA; every thread of
// the block calls it. False (for every thread) when the copy did not complete within the bound. Off the GPU (the CPU
// emulation of the kernels) thread 0 performs the same copy with the same zero fill.
__device__ bool StageTma(const CUtensorMap* map, uint64_t* bar, uint16_t* in, const uint16_t* frame, int H, int W,
                         int x, int y, int f, int rows, int cols)
{
#if defined(__CUDA_ARCH__)
	(void)frame; (void)H; (void)W;
	const uint32_t b = SmemAddr(bar);
	if (threadIdx.x == 0) {
		asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(b) : "memory");
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
		asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
		asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
		             :: "r"(b), "r"(static_cast<uint32_t>(rows * cols * 2)) : "memory");
		asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
		             :: "r"(SmemAddr(in)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(f), "r"(b)
		             : "memory");
	}
	__syncthreads();  // the barrier is initialised before any thread polls it
	bool ok = MbarWaitBounded(b, 0);
	const bool anyLate = __syncthreads_or(!ok);
	if (anyLate && !ok) { ok = MbarWaitBounded(b, 0); }  // the copy may still be in flight: wait for it once more
	if (threadIdx.x == 0) { asm volatile("mbarrier.inval.shared::cta.b64 [%0];" :: "r"(b) : "memory"); }
	return !anyLate;
#else
	(void)map; (void)bar;
	if (threadIdx.x == 0) {
		for (int r = 0; r < rows; ++r) {
			for (int c = 0; c < cols; ++c) {
				const int fy = y + r, fx = x + c;
				in[r * cols + c] = (fy >= 0 && fy < H && fx >= 0 && fx < W) ? frame[static_cast<long long>(fy) * W + fx] : 0;
			}
		}
	}
	(void)f;
	__syncthreads();
	return true;
#endif
}

// Replaces the zero-filled entries of a staged box (rows y.., columns x.., `rows` x `cols`, frame rows [0, H), columns
// [0, W)) by the nearest in-frame entry: first the columns outside the frame on every row, then the rows outside the
// frame as whole copies of the nearest in-frame row (read after the first step has completed it). Every read is of an
// entry the current step does not write. Ends with a block barrier when anything was replaced.
__device__ void StageFixBorders(uint16_t* in, int H, int W, int x, int y, int rows, int cols)
{
	const int nL = max(0, min(cols, -x)), nR = max(0, min(cols, x + cols - W));
	const int nT = max(0, min(rows, -y)), nB = max(0, min(rows, y + rows - H));
	if (nL + nR + nT + nB == 0) { return; }
	const int ncol = nL + nR;
	if (ncol > 0) {
		for (int idx = threadIdx.x; idx < rows * ncol; idx += blockDim.x) {
			const int r = idx / ncol, j = idx - r * ncol;
			const int c = j < nL ? j : cols - nR + (j - nL);
			const int src = min(max(x + c, 0), W - 1) - x;
			in[r * cols + c] = in[r * cols + src];
		}
		__syncthreads();
	}
	if (nT + nB > 0) {
		const int words = cols / 8;  // 16-byte words per row
		for (int idx = threadIdx.x; idx < (nT + nB) * words; idx += blockDim.x) {
			const int k = idx / words, v = idx - k * words;
			const int r = k < nT ? k : rows - nB + (k - nT);
			const int src = min(max(y + r, 0), H - 1) - y;
			reinterpret_cast<uint4*>(in + r * cols)[v] = reinterpret_cast<const uint4*>(in + src * cols)[v];
		}
		__syncthreads();
	}
}

__device__ __forceinline__ uint32_t Tap(uint32_t m2, uint32_t m1, uint32_t c, uint32_t p1, uint32_t p2)
{
	return 6u * c + 4u * (m1 + p1) + (m2 + p2);
}

// Bits 0-3 of m to the low bits of bytes 0-3 (the shifted copies 0, 7, 14, 21 do not overlap, so nothing carries).
__device__ __forceinline__ uint32_t Spread4(uint32_t m) { return (m * 0x00204081u) & 0x01010101u; }

// useTma: stage the input through the TMA with `map` (a tensor map of img as [frames][H][W]); otherwise with
// per-thread loads.
__global__ void __launch_bounds__(kThreads) DetectKernel(const uint16_t* __restrict__ img, Workspace ws, long long thrFixed,
                                                         const __grid_constant__ CUtensorMap map, int useTma)
{
	extern __shared__ __align__(16) unsigned char smemRaw[];
	// 128-byte aligned base (the TMA's shared-memory destination), whatever the dynamic area's own alignment
	unsigned char* base = smemRaw + ((128u - (SmemAddr(smemRaw) & 127u)) & 127u);
	uint32_t* c1 = reinterpret_cast<uint32_t*>(base);
	uint32_t* c2 = c1;
	uint32_t* v1 = c1 + kV1Off;
	__shared__ uint32_t scanSm[2 * kWarps + 2];
	__shared__ __align__(8) uint64_t tmaBar;
	const int H = ws.g.H, W = ws.g.W;
	const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, f = blockIdx.z;
	const uint16_t* frame = img + static_cast<long long>(f) * ws.g.N;
	const int tid = threadIdx.x;

	// stage the input tile (rows y0-7 .. y0+34, columns x0-8 .. x0+151, clamped into the frame) in the V1 space,
	// which pass B fills only after pass A: one TMA copy of the box and the border replication, or, without a tensor
	// map, every thread issues independent 16-byte loads when the tile's columns lie inside the frame and rows are
	// 16-byte aligned, clamped 2-byte loads otherwise (frame offsets fit in 32 bits)
	uint16_t* in = reinterpret_cast<uint16_t*>(v1);
	if (useTma) {
		if (!StageTma(&map, &tmaBar, in, frame, H, W, x0 - 8, y0 - 7, f, kInRows, kInW)) {
			if (tid == 0) { atomicExch(&ws.cnt->fault, 1u); }
			return;
		}
		StageFixBorders(in, H, W, x0 - 8, y0 - 7, kInRows, kInW);
	}
	else {
		const bool vec = x0 - 8 >= 0 && x0 - 8 + kInW <= W && (W & 7) == 0 &&
		                 (reinterpret_cast<uintptr_t>(frame) & 15) == 0;
		if (vec) {
			for (int q = tid; q < kInRows * (kInW / 8); q += kThreads) {
				const int r = q / (kInW / 8), v = q - r * (kInW / 8);
				const uint4* src = reinterpret_cast<const uint4*>(frame + clampi(y0 - 7 + r, 0, H - 1) * W + x0 - 8) + v;
				reinterpret_cast<uint4*>(in + r * kInW)[v] = __ldg(src);
			}
		}
		else {
			for (int q = tid; q < kInRows * kInW; q += kThreads) {
				const int r = q / kInW, c = q - r * kInW;
				in[q] = __ldg(frame + clampi(y0 - 7 + r, 0, H - 1) * W + clampi(x0 - 8 + c, 0, W - 1));
			}
		}
	}
	__syncthreads();
	// A: C1, one lane per column and run of rows (C1 column i = staged column i + 1); the three runs of a column
	// spread the 152 columns' work over all the block's threads
	for (int task = tid; task < kP1 * kRunsA; task += kThreads) {
		const int q = task / kP1, i = task - q * kP1;
		const int r0 = q * kRunA, r1 = min(kRows1, r0 + kRunA);
		const uint16_t* col = in + i + 1;
		uint32_t w0 = col[r0 * kInW], w1 = col[(r0 + 1) * kInW], w2 = col[(r0 + 2) * kInW], w3 = col[(r0 + 3) * kInW];
		#pragma unroll 4
		for (int r = r0; r < r1; ++r) {
			const uint32_t w4 = col[(r + 4) * kInW];
			c1[r * kP1 + i] = Tap(w0, w1, w2, w3, w4);
			w0 = w1; w1 = w2; w2 = w3; w3 = w4;
		}
	}
	__syncthreads();
	// B: V1, 4 columns per task from two 16-byte loads (consecutive tasks read and write consecutive 16-byte words,
	// so no two lanes of a quarter warp share a bank). C1 rows outside the frame are read at the nearest in-frame row:
	// the edge replication of the vertical pass.
	{
		const int rlo = max(0, 5 - y0), rhi = min(kRows1 - 1, H - 1 - y0 + 5);
		for (int task = tid; task < kRows1 * (kPV / 4); task += kThreads) {
			const int r = task / (kPV / 4), m = task - r * (kPV / 4);
			const int rs = min(max(r, rlo), rhi);
			const uint4* src = reinterpret_cast<const uint4*>(c1 + rs * kP1 + 4 * m);
			const uint4 a = src[0], b = src[1];
			const uint4 o = make_uint4(Tap(a.x, a.y, a.z, a.w, b.x), Tap(a.y, a.z, a.w, b.x, b.y), Tap(a.z, a.w, b.x, b.y, b.z),
			                           Tap(a.w, b.x, b.y, b.z, b.w));
			*reinterpret_cast<uint4*>(v1 + r * kPV + 4 * m) = o;
		}
	}
	__syncthreads();
	{
		// V1 columns outside the frame (the first clo and those after chi) take the nearest in-frame column's value;
		// only those columns are visited
		const int clo = max(0, 5 - x0), chi = min(kPV - 1, W - 1 - x0 + 5);
		const int ncol = clo + (kPV - 1 - chi);
		if (ncol > 0) {
			for (int idx = tid; idx < kRows1 * ncol; idx += kThreads) {
				const int r = idx / ncol, j = idx - r * ncol;
				const int i = j < clo ? j : chi + 1 + (j - clo);
				v1[r * kPV + i] = v1[r * kPV + (j < clo ? clo : chi)];
			}
			__syncthreads();
		}
	}
	// C: C2, one lane per column and run of up to 12 rows (C1 is dead: C2 takes its space)
	for (int task = tid; task < kPV * 3; task += kThreads) {
		const int q = task / kPV, i = task - q * kPV;
		const int r0 = 12 * q, nr = min(12, kRows2 - r0);
		uint32_t v[20];
		#pragma unroll
		for (int t = 0; t < 20; ++t) { v[t] = t < nr + 8 ? v1[(r0 + t) * kPV + i] : 0u; }
		#pragma unroll
		for (int t = 0; t < 12; ++t) {
			if (t < nr) { c2[(r0 + t) * kPV + i] = Tap(v[t], v[t + 2], v[t + 4], v[t + 6], v[t + 8]); }
		}
	}
	__syncthreads();
	// D: W1 on the ring, in place of V1, 4 ring columns per task (three 16-byte loads of C2, one of V1, one store;
	// consecutive tasks on consecutive 16-byte words)
	for (int task = tid; task < kRows2 * kTasksD; task += kThreads) {
		const int q = task / kTasksD, m = task - q * kTasksD;
		const uint4* src = reinterpret_cast<const uint4*>(c2 + q * kPV + 4 * m);
		const uint4 a = src[0], b = src[1], c = src[2];
		const uint32_t u[12] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
		uint4* vp = reinterpret_cast<uint4*>(v1 + (q + 4) * kPV + 4 * m + 4);
		const uint4 e = *vp;
		const uint32_t v[4] = {e.x, e.y, e.z, e.w};
		const int y = y0 + q - 1, xs = x0 + 4 * m - 1;
		const bool rowIn = y >= 0 && y < H;
		uint32_t o[4];
		if (rowIn && xs >= 0 && xs + 4 <= W) {
			// all four inside the frame: max(W1, 0) = max(V1 * 256, V2) - V2
			#pragma unroll
			for (int k = 0; k < 4; ++k) {
				const uint32_t v2 = Tap(u[k], u[k + 2], u[k + 4], u[k + 6], u[k + 8]);
				o[k] = max(v[k] << 8, v2) - v2;
			}
		}
		else {
			#pragma unroll
			for (int k = 0; k < 4; ++k) {
				const uint32_t v2 = Tap(u[k], u[k + 2], u[k + 4], u[k + 6], u[k + 8]);
				const uint32_t v1s = v[k] << 8;
				const int x = xs + k;
				o[k] = (rowIn && x >= 0 && x < W && v1s > v2) ? v1s - v2 : 0u;
			}
		}
		*vp = make_uint4(o[0], o[1], o[2], o[3]);
	}
	__syncthreads();
	// E: domain and seeds, 4 pixels per task (a warp covers one tile row: consecutive 16-byte loads), up to four
	// tasks per thread; the masks of the thread's tasks are packed 4 bits per task
	const uint32_t thr = thrFixed <= 0 ? 0u : (thrFixed >= 0xffffffffll ? 0xffffffffu : static_cast<uint32_t>(thrFixed));
	uint32_t dmask = 0, smask = 0;
	#pragma unroll
	for (int h = 0; h < kTasksE; ++h) {
		const int task = tid + h * kThreads;
		const int ty = task >> 5, m = task & 31;
		if (ty >= TY) { continue; }  // 32 tasks per tile row; the last thread slots have none
		uint32_t a[3][8];
		#pragma unroll
		for (int rr = 0; rr < 3; ++rr) {
			const uint4* src = reinterpret_cast<const uint4*>(v1 + (ty + 4 + rr) * kPV + 4 * m + 4);
			const uint4 p = src[0], q = src[1];
			a[rr][0] = p.x; a[rr][1] = p.y; a[rr][2] = p.z; a[rr][3] = p.w;
			a[rr][4] = q.x; a[rr][5] = q.y; a[rr][6] = q.z; a[rr][7] = q.w;
		}
		// 3 x 3 maximum as column maxima, then the maximum of three of them; a seed is not below the maximum of its
		// window, which holds the pixel itself, so this equals "no neighbour strictly greater"
		uint32_t cm[6];
		#pragma unroll
		for (int j = 0; j < 6; ++j) { cm[j] = __vimax3_u32(a[0][j], a[1][j], a[2][j]); }
		const int inFrame = y0 + ty < H ? W - (x0 + 4 * m) : 0;  // pixels k < inFrame lie inside the frame
		#pragma unroll
		for (int k = 0; k < 4; ++k) {
			const uint32_t v = a[1][k + 1];
			const bool dom = k < inFrame && v > thr;
			dmask |= static_cast<uint32_t>(dom) << (4 * h + k);
			smask |= static_cast<uint32_t>(dom && v >= __vimax3_u32(cm[k], cm[k + 1], cm[k + 2])) << (4 * h + k);
		}
	}
	// block-wide positions in the domain and seed lists: one atomic per list, issued by thread 0 while the other
	// threads write the code bytes and the W1 of domain pixels, which need no list position
	const int lane = tid & 31, warp = tid >> 5;
	const uint32_t nd = __popc(dmask), ns = __popc(smask);
	uint32_t id = nd, is = ns;
	#pragma unroll
	for (int d = 1; d < 32; d <<= 1) {
		const uint32_t td = __shfl_up_sync(0xffffffffu, id, d), ts = __shfl_up_sync(0xffffffffu, is, d);
		if (lane >= d) { id += td; is += ts; }
	}
	if (lane == 31) { scanSm[warp] = id; scanSm[kWarps + warp] = is; }
	__syncthreads();
	if (tid == 0) {
		uint32_t sd = 0, ss = 0;
		for (int w = 0; w < kWarps; ++w) {
			const uint32_t a = scanSm[w], b = scanSm[kWarps + w];
			scanSm[w] = sd; scanSm[kWarps + w] = ss;
			sd += a; ss += b;
		}
		scanSm[2 * kWarps] = sd ? atomicAdd(&ws.cnt->ndom, sd) : 0u;
		scanSm[2 * kWarps + 1] = ss ? atomicAdd(&ws.cnt->nseed, ss) : 0u;
		// per-frame counts: the watershed's exactness bound and the lists of frames flooded again frame-wide
		if (sd) { atomicAdd(ws.frameDom + f, sd); }
		if (ss) { atomicAdd(ws.frameSeeds + f, ss); }
	}
	// code bytes of the four pixels of each task and the W1 of its domain pixels (still in shared memory); a chunk's
	// pixel indices fit in 31 bits
	const uint32_t frameBase = static_cast<uint32_t>(f) * static_cast<uint32_t>(ws.g.N);
	#pragma unroll
	for (int h = 0; h < kTasksE; ++h) {
		const int task = tid + h * kThreads;
		const int ty = task >> 5, m = task & 31;
		const int y = y0 + ty, xb = x0 + 4 * m;
		if (ty >= TY || y >= H || xb >= W) { continue; }
		const uint32_t g = frameBase + static_cast<uint32_t>(y * W + xb);
		// each mask bit spread to the low bit of its byte, times the flag
		const uint32_t dm = (dmask >> (4 * h)) & 15u, sm = (smask >> (4 * h)) & 15u;
		const uint32_t bytes = Spread4(dm) * kDomain | Spread4(sm) * kSeed;
		if (xb + 4 <= W && (g & 3u) == 0) { *reinterpret_cast<uint32_t*>(ws.code + g) = bytes; }
		else {
			for (int k = 0; k < 4 && xb + k < W; ++k) { ws.code[g + k] = static_cast<uint8_t>(bytes >> (8 * k)); }
		}
		const uint32_t* w1row = v1 + (ty + 5) * kPV + 4 * m + 5;
		#pragma unroll
		for (int k = 0; k < 4; ++k) {
			if ((dm >> k) & 1u) { ws.w1[g + k] = w1row[k]; }
		}
	}
	__syncthreads();
	// the list entries, lowest pixel first
	uint32_t pd = scanSm[2 * kWarps] + scanSm[warp] + id - nd;
	uint32_t ps = scanSm[2 * kWarps + 1] + scanSm[kWarps + warp] + is - ns;
	#pragma unroll
	for (int h = 0; h < kTasksE; ++h) {
		const uint32_t dm = (dmask >> (4 * h)) & 15u, sm = (smask >> (4 * h)) & 15u;
		if ((dm | sm) == 0) { continue; }  // also every task outside the tile or the frame (its masks are empty)
		const int task = tid + h * kThreads;
		const int ty = task >> 5, m = task & 31;
		const uint32_t g = frameBase + static_cast<uint32_t>((y0 + ty) * W + x0 + 4 * m);
		for (uint32_t b = dm; b; b &= b - 1u) {
			if (pd < ws.capDom) { ws.dom[pd] = g + static_cast<uint32_t>(__ffs(b) - 1); }
			else { atomicExch(&ws.cnt->overflow, 1u); }
			++pd;
		}
		for (uint32_t b = sm; b; b &= b - 1u) {
			if (ps < ws.capSeed) { ws.seeds[ps] = g + static_cast<uint32_t>(__ffs(b) - 1); }
			else { atomicExch(&ws.cnt->overflow, 1u); }
			++ps;
		}
	}
}

// One wavelet plane as float64 (level 0: W0 = V0 - V1, 1: W1 = V1 - V2, 2: residual V2), for the Wavelett export.
__global__ void __launch_bounds__(kThreads) PlaneKernel(const uint16_t* __restrict__ img, double* __restrict__ out,
                                                        int H, int W, long long N, int level)
{
	extern __shared__ __align__(16) unsigned char smemRaw[];
	TileSmem& s = *reinterpret_cast<TileSmem*>(smemRaw);
	const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, f = blockIdx.z;
	const uint16_t* frame = img + static_cast<long long>(f) * N;
	WaveletTile(s, frame, H, W, x0, y0);
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	for (int ty = warp; ty < TY; ty += kWarps) {
		const int y = y0 + ty;
		if (y >= H) { continue; }
		for (int tx = lane; tx < TX; tx += 32) {
			const int x = x0 + tx;
			if (x >= W) { continue; }
			double val;
			if (level == 0) {
				// W0 = in - V1, in units of 1/256 (the input tile buffer now holds V1: read the pixel itself)
				const long long d = static_cast<long long>(__ldg(frame + static_cast<long long>(y) * W + x)) * 256 - s.a.v1[ty + 5][tx + 5];
				val = static_cast<double>(d) * (1.0 / 256.0);
			}
			else if (level == 1) { val = static_cast<double>(W1At(s, ty + 1, tx + 1)) * kW1Unit; }
			else { val = static_cast<double>(s.v2[ty + 1][tx + 1]) * kW1Unit; }
			out[static_cast<long long>(f) * N + static_cast<long long>(y) * W + x] = val;
		}
	}
}

// Once per process (a function-local static is initialised once, also when several threads call at the same time).
bool ConfigureSmem()
{
	static const bool done = [] {
		const int bytes = static_cast<int>(sizeof(TileSmem));
		bool ok = PTB_CUDA(cudaFuncSetAttribute(DetectKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kDetectBytes));
		return ok && PTB_CUDA(cudaFuncSetAttribute(PlaneKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
	}();
	return done;
}

// The driver's tensor-map encoder (cuTensorMapEncodeTiled), fetched once through the runtime so that the library
// needs no link against the driver library; null when unavailable or when PTB_DETECT_TMA=0 selects the per-thread
// staging loads.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn TensorMapEncoder()
{
	static const EncodeTiledFn fn = []() -> EncodeTiledFn {
		if (const char* e = std::getenv("PTB_DETECT_TMA")) {
			if (std::atoi(e) == 0) { return nullptr; }
		}
		void* p = nullptr;
		cudaDriverEntryPointQueryResult q{};
		if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
		    q != cudaDriverEntryPointSuccess) {
			cudaGetLastError();
			return nullptr;
		}
		return reinterpret_cast<EncodeTiledFn>(p);
	}();
	return fn;
}

// Tensor map of a chunk's frames for the detection kernel's input box; false when the TMA cannot describe them
// (width not a multiple of 8, base not 16-byte aligned) or the encoder refuses, and the kernel then stages with
// per-thread loads.
bool EncodeInputMap(CUtensorMap& map, const uint16_t* img, int H, int W, int B)
{
	const EncodeTiledFn enc = TensorMapEncoder();
	if (enc == nullptr || (W & 7) != 0 || (reinterpret_cast<uintptr_t>(img) & 15) != 0 || B < 1) { return false; }
	const cuuint64_t dims[3] = {static_cast<cuuint64_t>(W), static_cast<cuuint64_t>(H), static_cast<cuuint64_t>(B)};
	const cuuint64_t strides[2] = {static_cast<cuuint64_t>(W) * 2, static_cast<cuuint64_t>(W) * H * 2};
	const cuuint32_t box[3] = {kInW, kInRows, 1};
	const cuuint32_t elem[3] = {1, 1, 1};
	return enc(&map, CU_TENSOR_MAP_DATA_TYPE_UINT16, 3, const_cast<uint16_t*>(img), dims, strides, box, elem,
	           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
	           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

// thr is compared as W1_fixed > floor(thr * 2^16); thresholds beyond the W1 range (|W1| < 2^33) or NaN saturate.
long long ThresholdFixed(double thr)
{
	const double t = std::floor(thr * 65536.0);
	if (!(t < 4.0e18)) { return 4000000000000000000ll; }  // +large, +inf and NaN: nothing passes
	if (t < -4.0e18) { return -4000000000000000000ll; }
	return static_cast<long long>(t);
}

namespace {
std::atomic<uint64_t> g_detectStaging[2];  // detection launches staged by the TMA, by per-thread loads
}  // namespace

void DetectStagingStats(uint64_t* out, int n)
{
	for (int k = 0; k < 2; ++k) {
		const uint64_t v = g_detectStaging[k].exchange(0);
		if (k < n) { out[k] = v; }
	}
}

bool LaunchDetect(const Workspace& ws, double thr, cudaStream_t st)
{
	if (!ConfigureSmem()) { return false; }
	const dim3 grid((ws.g.W + TX - 1) / TX, (ws.g.H + TY - 1) / TY, ws.g.B);
	CUtensorMap map;
	std::memset(&map, 0, sizeof(map));
	const int useTma = EncodeInputMap(map, ws.img, ws.g.H, ws.g.W, ws.g.B) ? 1 : 0;
	DetectKernel<<<grid, kThreads, kDetectBytes, st>>>(ws.img, ws, ThresholdFixed(thr), map, useTma);
	g_detectStaging[useTma ? 0 : 1].fetch_add(1);
	CountLaunch();
	return PTB_LAUNCHED();
}

bool LaunchPlane(const uint16_t* img, double* out, int H, int W, int B, int level, cudaStream_t st)
{
	if (!ConfigureSmem()) { return false; }
	const dim3 grid((W + TX - 1) / TX, (H + TY - 1) / TY, B);
	PlaneKernel<<<grid, kThreads, sizeof(TileSmem), st>>>(img, out, H, W, static_cast<long long>(H) * W, level);
	CountLaunch();
	return PTB_LAUNCHED();
}

}  // namespace ptb
