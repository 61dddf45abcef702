// Fit-only entry point that allocates no device memory, for callers that cannot call cudaMalloc.
//
// Who needs it: code that runs where device allocation is not available or not allowed - inside a host callback or a
// stream-ordered pipeline owned by another runtime, under an allocator that hands out only pre-sized pools, or in a
// process whose device memory budget is fixed before this library is loaded. Such callers bring their own device
// buffers for the stack, the positions and the output rows; everything else the fit needs (the per-point fit inputs,
// per-plane counters for the Index column, re-fit flags) lives in one static device array defined in this file.
//
// Limits and behaviour:
//   * at most kNoAllocMaxPoints points and kNoAllocMaxPlanes planes per call; larger calls are rejected (error);
//   * fit modes 0-4, 6 and 7 (modes 5 and 8 need their coefficient table in device memory and are rejected);
//   * the static array is shared by every call on a device and keeps the previous call's contents; the counters are
//     cleared at the start of each call; calls that overlap on the GPU (e.g. issued on two streams) race on it;
//   * every GPU that loads the library holds the array (about 3 MB) until the process exits;
//   * the first call on a device looks up the array's device address (cudaGetSymbolAddress) with that device current.
#include <mutex>

#include "engine.h"

namespace ptb {

bool LaunchFit(const uint16_t* img, int H, int W, long long N, const Cand* cands, const uint32_t* nptr, uint32_t nconst,
               uint32_t cap, const FitParams& fp, double* rows, uint8_t* flags, int precision, cudaStream_t st);

namespace {

constexpr uint32_t kNoAllocMaxPoints = 65536;
constexpr uint32_t kNoAllocMaxPlanes = 65536;

struct NoAllocScratch {
	Cand cand[kNoAllocMaxPoints];
	uint32_t localIndex[kNoAllocMaxPoints];
	uint32_t planeCount[kNoAllocMaxPlanes];
	uint8_t flags[kNoAllocMaxPoints];
	unsigned int fallbacks;
	unsigned int mleQueue[2];  // work-queue counters of the persistent fit kernels (zeroed by the fit launch)
};

// The scratch. In host code this name is only a stand-in for the symbol, never a device address: kernels receive
// the address that cudaGetSymbolAddress returns for the current device.
static __device__ __align__(256) unsigned char g_noAllocScratch[sizeof(NoAllocScratch)];

// positions -> fit inputs; rows with a plane outside the stack get a position that fails the border test (the same
// convention as the host Fitting path)
__global__ void NoAllocPrepare(const double* __restrict__ pos, uint32_t n, uint64_t planes, NoAllocScratch* s)
{
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		const double* p = pos + static_cast<size_t>(i) * 6;
		Cand c;
		c.x = p[2];
		c.y = p[3];
		c.intensity = p[4];
		c.surf = p[5];
		c.image = 0;
		const double pl = p[1];
		if (!(pl >= 1.0) || static_cast<uint64_t>(pl) > planes) {
			c.x = -1.0;
			c.y = -1.0;
			c.frame = 0;
		}
		else { c.frame = static_cast<int>(static_cast<uint64_t>(pl) - 1); }
		s->cand[i] = c;
	}
}

// Index column: rank of each point among the earlier points of its plane (input order), 1-based. One warp walks the
// points 32 at a time; lanes that share a plane are ranked with a match mask.
__global__ void NoAllocIndex(const double* __restrict__ pos, uint32_t n, uint64_t planes, NoAllocScratch* s)
{
	const int lane = threadIdx.x & 31;
	for (uint64_t p = lane; p < planes; p += 32) { s->planeCount[p] = 0; }
	if (lane == 0) { s->fallbacks = 0; }
	__syncwarp();
	for (uint32_t base = 0; base < n; base += 32) {
		const uint32_t i = base + lane;
		const bool active = i < n;
		const double pl = active ? pos[static_cast<size_t>(i) * 6 + 1] : 0.0;
		const bool valid = active && pl >= 1.0 && static_cast<uint64_t>(pl) <= planes;
		const uint32_t key = valid ? static_cast<uint32_t>(static_cast<uint64_t>(pl) - 1) : 0xffffffffu;
		const unsigned same = __match_any_sync(0xffffffffu, key);
		const unsigned below = same & ((1u << lane) - 1u);
		uint32_t idx = 0;
		if (valid) { idx = s->planeCount[key] + __popc(below) + 1; }
		__syncwarp();
		// the highest lane of each plane group publishes the new count
		if (valid && (same >> lane) == 1u) { s->planeCount[key] = idx; }
		if (active) { s->localIndex[i] = idx; }
		__syncwarp();
	}
}

__global__ void NoAllocFinish(const double* __restrict__ pos, uint32_t n, uint64_t planes, const NoAllocScratch* s, double* rows)
{
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		const double* p = pos + static_cast<size_t>(i) * 6;
		double* r = rows + static_cast<size_t>(i) * kCols;
		const double pl = p[1];
		if (!(pl >= 1.0) || static_cast<uint64_t>(pl) > planes) {
			r[cX] = p[2];
			r[cY] = p[3];
		}
		r[cId] = p[0];
		r[cPlane] = p[1];
		r[cIndex] = static_cast<double>(s->localIndex[i]);
	}
}

std::mutex g_addrMutex;
void* g_addr[64] = {};

// Device address of the scratch for the current device, looked up once per device with that device current.
NoAllocScratch* ScratchForCurrentDevice()
{
	int dev = 0;
	if (!PTB_CUDA(cudaGetDevice(&dev)) || dev < 0 || dev >= 64) { return nullptr; }
	std::lock_guard<std::mutex> lock(g_addrMutex);
	if (g_addr[dev] == nullptr) {
		void* ptr = nullptr;
		if (!PTB_CUDA(cudaGetSymbolAddress(&ptr, g_noAllocScratch))) { return nullptr; }
		g_addr[dev] = ptr;
	}
	return static_cast<NoAllocScratch*>(g_addr[dev]);
}

}  // namespace

// Returns doubles written (nPoints * 18), 0 for an empty call, -1 on error (message recorded).
long long FittingDeviceNoAlloc(const uint16_t* dStack, const double* dPositions, uint64_t nPoints, double* dOutput,
                               uint64_t height, uint64_t width, uint64_t planes, uint64_t fit, const double* fitParams,
                               int precision, int lanes, cudaStream_t st)
{
	if (nPoints == 0) { return 0; }
	if (nPoints > kNoAllocMaxPoints) {
		SetError("PTB_FittingDeviceNoAlloc: at most " + std::to_string(kNoAllocMaxPoints) + " points per call");
		return -1;
	}
	if (planes > kNoAllocMaxPlanes) {
		SetError("PTB_FittingDeviceNoAlloc: at most " + std::to_string(kNoAllocMaxPlanes) + " planes per call");
		return -1;
	}
	if (fit == kSplineEmccd || fit == kMleSpline) {
		SetError("PTB_FittingDeviceNoAlloc: spline modes 5 and 8 are not available without device allocation");
		return -1;
	}
	// each dimension is bounded before the product is formed, so the product cannot wrap
	constexpr uint64_t kMaxPixels = (1ull << 31) - 1;
	if (height == 0 || width == 0 || planes == 0 || height > kMaxPixels || width > kMaxPixels || height > kMaxPixels / width) {
		SetError("PTB_FittingDeviceNoAlloc: invalid stack dimensions");
		return -1;
	}
	FitParams fp;
	std::vector<double> unused;
	if (!ParseFitParams(fit, fitParams, fp, unused)) { return -1; }
	NoAllocScratch* s = ScratchForCurrentDevice();
	if (s == nullptr) { return -1; }
	fp.mle.fallbacks = &s->fallbacks;
	fp.mle.queue = s->mleQueue;
	fp.lanes = lanes;
	// modes 6-8: the ROI mapping the Fitting export picks for the same call (a warp per ROI while the points fill the
	// GPU a few times at most, else a thread per ROI), so that both give the same rows
	if (fp.mode >= kMleGauss && fp.lanes == 0) { fp.lanes = nPoints <= 148ull * 64 ? 32 : 1; }
	const uint32_t n = static_cast<uint32_t>(nPoints);
	const uint32_t blocks = std::min<uint32_t>((n + 255) / 256, 148u * 4u);
	NoAllocPrepare<<<blocks, 256, 0, st>>>(dPositions, n, planes, s);
	NoAllocIndex<<<1, 32, 0, st>>>(dPositions, n, planes, s);
	CountLaunch(2);
	if (!PTB_LAUNCHED()) { return -1; }
	const int H = static_cast<int>(height), W = static_cast<int>(width);
	if (!LaunchFit(dStack, H, W, static_cast<long long>(height) * width, s->cand, nullptr, n, n, fp, dOutput, s->flags,
	               precision, st)) {
		return -1;
	}
	NoAllocFinish<<<blocks, 256, 0, st>>>(dPositions, n, planes, s, dOutput);
	CountLaunch();
	if (!PTB_LAUNCHED()) { return -1; }
	return static_cast<long long>(nPoints) * kCols;
}

}  // namespace ptb
