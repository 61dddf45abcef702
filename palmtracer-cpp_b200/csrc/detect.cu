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
//   W1 = V1 * 256 - V2        (units 2^-16, |W1| < 2^32, int64)
// with h' = {1, 4, 6, 4, 1}. Each pass evaluates its output at the CLAMPED coordinate, exactly like the reference's
// offsetTest() clamping of every neighbour access, so border tiles need no special case. The strict threshold
// W1 > thr is evaluated as W1_fixed > floor(thr * 2^16), which is the same test for an integer W1_fixed.
//
// Layout: a 128 x 32 output tile per CTA of 8 warps; every stage loops rows over warps and columns over lanes (no
// index division); shared buffers are reused across stages (input -> V1, T1 -> T2), 66 KB in all.
#include <algorithm>
#include <cmath>

#include "pt_common.cuh"

namespace ptb {

namespace {

constexpr int TX = 128, TY = 32;          // output tile
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

// Appends `g` to list[] for every lane with pred set: one atomic per warp. Entries beyond cap raise *overflow.
__device__ __forceinline__ void WarpAppend(bool pred, uint32_t g, uint32_t* list, uint32_t* counter, uint32_t cap,
                                           uint32_t* overflow)
{
	const unsigned mask = __ballot_sync(0xffffffffu, pred);
	if (mask == 0) { return; }
	const int lane = threadIdx.x & 31;
	const int leader = __ffs(mask) - 1;
	uint32_t base = 0;
	if (lane == leader) { base = atomicAdd(counter, static_cast<uint32_t>(__popc(mask))); }
	base = __shfl_sync(0xffffffffu, base, leader);
	if (pred) {
		const uint32_t pos = base + __popc(mask & ((1u << lane) - 1u));
		if (pos < cap) { list[pos] = g; }
		else { atomicExch(overflow, 1u); }
	}
}

// One CTA per (tile, frame): W1, domain and seed flags for the tile; W1 stored on domain pixels only.
__global__ void __launch_bounds__(kThreads) DetectKernel(const uint16_t* __restrict__ img, Workspace ws, long long thrFixed)
{
	extern __shared__ __align__(16) unsigned char smemRaw[];
	TileSmem& s = *reinterpret_cast<TileSmem*>(smemRaw);
	const int H = ws.g.H, W = ws.g.W;
	const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, f = blockIdx.z;
	const uint16_t* frame = img + static_cast<long long>(f) * ws.g.N;
	WaveletTile(s, frame, H, W, x0, y0);
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const long long thr = thrFixed > 0 ? thrFixed : 0;  // domain: W1 > thr and W1 > 1e-8, i.e. W1_fixed >= 1
	// every thread visits the same number of pixels (uniform for the warp-wide appends)
	for (int ty = warp; ty < TY; ty += kWarps) {
		const int y = y0 + ty;
		for (int tx = lane; tx < TX; tx += 32) {
			const int x = x0 + tx;
			const bool inside = y < H && x < W;
			bool domain = false, seed = false;
			long long v = 0;
			if (inside) {
				v = W1At(s, ty + 1, tx + 1);
				domain = v > thr;
				if (domain) {
					seed = true;
					// a neighbour dominates only if its thresholded value is strictly larger; since v > thr, that is
					// exactly W1(neighbour) > W1(pixel)
					for (int dy = -1; dy <= 1; ++dy) {
						const int yy = y + dy;
						if (yy < 0 || yy >= H) { continue; }
						for (int dx = -1; dx <= 1; ++dx) {
							const int xx = x + dx;
							if ((dx == 0 && dy == 0) || xx < 0 || xx >= W) { continue; }
							if (W1At(s, ty + 1 + dy, tx + 1 + dx) > v) { seed = false; }
						}
					}
				}
			}
			const long long gl = static_cast<long long>(f) * ws.g.N + static_cast<long long>(y) * W + x;
			if (inside) {
				ws.code[gl] = static_cast<uint8_t>((domain ? kDomain : 0) | (seed ? kSeed : 0));
				if (domain) { ws.w1[gl] = v; }
			}
			WarpAppend(domain, static_cast<uint32_t>(gl), ws.dom, &ws.cnt->ndom, ws.capDom, &ws.cnt->overflow);
			WarpAppend(seed, static_cast<uint32_t>(gl), ws.seeds, &ws.cnt->nseed, ws.capSeed, &ws.cnt->overflow);
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

bool ConfigureSmem()
{
	static bool done = false;
	if (done) { return true; }
	const int bytes = static_cast<int>(sizeof(TileSmem));
	bool ok = PTB_CUDA(cudaFuncSetAttribute(DetectKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
	ok = ok && PTB_CUDA(cudaFuncSetAttribute(PlaneKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
	done = ok;
	return ok;
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

bool LaunchDetect(const Workspace& ws, double thr, cudaStream_t st)
{
	if (!ConfigureSmem()) { return false; }
	const dim3 grid((ws.g.W + TX - 1) / TX, (ws.g.H + TY - 1) / TY, ws.g.B);
	DetectKernel<<<grid, kThreads, sizeof(TileSmem), st>>>(ws.img, ws, ThresholdFixed(thr));
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
