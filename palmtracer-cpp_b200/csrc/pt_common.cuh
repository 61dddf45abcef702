// Shared definitions of the B200 localization engine: constants of the reference algorithm, error plumbing and
// the device workspace layout of one chunk of frames.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>

namespace ptb {

// ---- Constants of the reference algorithm (lib/Constants.hpp:20-24, 53; Segmentation2D.hpp:80; Fitting.hpp:80)
constexpr int kCols = 18;            // columns of one localization row
constexpr double kEps = 1e-7;        // EPSILON: watershed aging step and fill() guards
constexpr double kSeedFloor = 1e-8;  // potentials above this join the watershed domain
constexpr double kVolumeMin = 4;     // a region needs surf > 4
constexpr int kMaxIter = 75;         // LM iteration cap
constexpr int kThresholdIters = 5;   // AutoThreshold rounds

// Column indices (lib/Constants.hpp:31-51)
enum Col : int {
	cId = 0, cPlane, cIndex, cChannel, cX, cY, cZ, cIntensity, cSigmaX, cSigmaY, cTheta,
	cQualityXY, cQualityZ, cAmplitude, cOffset, cSegIntensity, cSurface, cCircularity
};

// Fit modes (lib/fit/Fitting.hpp:22-30)
enum FitMode : int { kNone = 0, kG2Fixed = 1, kG2Sigma = 2, kG3Fixed = 3, kG3Theta = 4, kSplineEmccd = 5,
                     kMleGauss = 6, kMleAstig = 7, kMleSpline = 8 };

// Per-pixel code byte written by the detection kernel.
constexpr uint8_t kDomain = 1;  // thresholded potential > 1e-8: the watershed floods it
constexpr uint8_t kSeed = 2;    // local maximum of the thresholded potential
constexpr int kDirShift = 2;    // bits 2..4: raster-earlier seed neighbour a seed inherits its label from (0 = root)

// Rank test of the per-component floods: at most kRankSlots frames per chunk, kSuspectCap boundary pairs per chunk
// and kPairsPerFrame per frame (a frame beyond these limits is flooded again frame-wide instead).
constexpr uint32_t kRankSlots = 64u;
constexpr uint32_t kSuspectCap = 16384u;
constexpr uint32_t kPairsPerFrame = 512u;
// Re-flood of the frames that fail the rank test: at most kRefloodSlots frames per chunk, each with at most
// kRefloodCap domain pixels (their W1 values are grouped by value bucket for the rank lookups); other frames are
// flooded frame-wide.
constexpr uint32_t kRefloodSlots = 8u;
constexpr uint32_t kRefloodCap = 65536u;
constexpr uint32_t kRefloodBuckets = 32768u;  // value buckets of the rank lookups
// Words per pixel and re-flood slot of rfPix: the estimated frame-wide pop position, its bound B, and for groups
// re-flooded in global memory (larger than the shared-memory box) the element value and its chain minimum (int64
// each).
constexpr uint32_t kRfWords = 6u;

// W1 values are exact multiples of 2^-16 (B3 taps are dyadic and the input is uint16), kept as int64 "fixed" units.
constexpr double kW1Unit = 1.0 / 65536.0;

// Component id tag stored in par[root] once components are enumerated.
constexpr uint32_t kCompTag = 0x80000000u;

// ---- Error plumbing: no exception crosses the C ABI; the first failure of a call is recorded per thread.
void SetError(const std::string& msg);
const std::string& LastError();
void ClearError();
bool CheckCuda(cudaError_t e, const char* what, const char* file, int line);
void CountLaunch(uint64_t n = 1);

#define PTB_CUDA(call) ::ptb::CheckCuda((call), #call, __FILE__, __LINE__)
#define PTB_LAUNCHED() ::ptb::CheckCuda(cudaGetLastError(), "kernel launch", __FILE__, __LINE__)

// ---- Device counters of one chunk (one struct in device memory, read back once per chunk).
struct Counters {
	uint32_t ndom;      // domain pixels appended to dom[]
	uint32_t nseed;     // seed pixels appended to seeds[]
	uint32_t ncomp;     // connected components of the domain
	uint32_t nmulti;    // components holding more than one region
	uint32_t nregion;   // regions (root seeds)
	uint32_t ncand;     // regions with surf > 4
	uint32_t nfit;      // candidates kept under the per-plane capacity
	uint32_t overflow;  // a list outgrew its capacity (the chunk must be redone with room)
	uint32_t truncated; // some plane had more candidates than the per-plane capacity
	uint32_t refit;     // FP32 fits redone in FP64
	uint32_t nroute;    // frames whose per-component flood could differ from the frame-wide one (flooded again)
	uint32_t queue[2];  // work-queue counters of the persistent fit kernels
	uint32_t nsuspect;  // boundary pairs that failed the flood's first exactness test (kept for the rank test)
	uint32_t nslots;    // frames given the rank test
	uint32_t nreflood;  // frames that failed the rank test (flooded again with estimated frame-wide aging)
	uint32_t nrfgroup;  // multi-label groups of the frames given a re-flood slot (listed in rfGroups)
	uint32_t routeWhy[7];  // frames flooded frame-wide, by the first reason (RouteReason)
	uint32_t fault;        // a kernel's bounded wait ran out (its results are void; the call fails)
	uint32_t boxNext;      // work queue of the shared-memory group floods: next multi-label group to take
	uint32_t nunion;       // domain pixels that join two union-find trees (listed in lab for the union pass)
};

// Why a frame is flooded again frame-wide (diagnostics, counted per frame by the first reason).
enum RouteReason : int {
	kRouteSuspectFull = 0,  // the list of boundary pairs that failed the first test was full
	kRouteFirstTest = 1,    // a pair failed the first test where no rank test follows (segmentation mode 2)
	kRouteRankSlots = 2,    // more frames needed the rank test than a chunk has slots
	kRoutePairs = 3,        // the frame had more failing pairs than the rank test takes per frame
	kRouteRankFused = 4,    // failed the rank test after a basin fusion (no re-flood)
	kRouteRefloodSlots = 5, // failed the rank test beyond the re-flood slots or the re-flood's domain-pixel capacity
	kRouteRefloodTest = 6   // the re-flooded labels failed the per-element rank test
};

// One fit input: a segmentation candidate (x_, y_, intensity_, surf_ of SegmentationInfo) or a caller position.
struct Cand {
	double x, y, intensity, surf;
	int frame;  // plane within the device stack the ROI is read from
	int image;  // entry of the launch's FitImages holding that stack (0 unless a launch fuses several stacks)
};

// The device stacks a maximum-likelihood fit launch reads: one, or several when the serving layer fuses the
// candidates of concurrent requests into one launch (Cand::image selects the entry).
constexpr int kMaxFitImages = 16;
struct FitImage {
	const uint16_t* img;
	int H, W;
	long long N;  // H * W
};
struct FitImages {
	int n;
	FitImage im[kMaxFitImages];
};
inline FitImages OneImage(const uint16_t* img, int H, int W, long long N)
{
	FitImages f{};
	f.n = 1;
	f.im[0] = FitImage{img, H, W, N};
	return f;
}

// Maximum-likelihood modes 6-8 (fit_params layouts in include/palmtracer_b200.h).
struct MleParams {
	int model, roi, half, n, maxIter;
	int chunk;  // candidates taken from the persistent kernels' work queue at a time (0 or 1: one)
	double sigma0, offset, gain, crlbMax, pixelSize, zMin, zMax;
	double astig[10];
	int sx, sy, sz;
	double dz;
	const float* table;        // mode 8: cell-major [cell][64], FP32 (FP32 phases)
	const double* table64;     // mode 8: the same in FP64 (FP64 phases)
	unsigned int* fallbacks;   // FP64 Cholesky re-factorisations (diagnostics)
	unsigned int* queue;       // 2 work-queue counters of the persistent fit kernels (zeroed by the launch), or null
	unsigned long long* evals; // profiling, or null: model evaluations [FP32 LM, FP32 polish, FP64 pre-scan + final]
};

// Fit configuration passed by value to the fit kernels.
struct FitParams {
	int mode;        // FitMode
	int roi;         // forced odd
	int half;
	int n;           // roi * roi
	int nParams;
	double sigmaX, sigmaY, theta;
	// spline (mode 5)
	int sx, sy, sz;
	long long splineSize;  // sx * sy * sz
	long long offsetXY;
	double roiParam, initZ, deltaZ, intensityRatio;
	const double* coeffs;  // device, cell-major [cell][64]
	MleParams mle;         // modes 6-8
	int lanes;             // ROI mapping for modes 6-8: 1 thread per ROI, else warp per ROI (autotuned)
	cudaEvent_t* marks;    // profiling, or null: 5 events recorded around the phases of the modes 6-8 fit
};

// Division of a 31-bit unsigned value by a fixed divisor d >= 1 as one multiply and a shift (division by invariant
// integers, Granlund and Montgomery 1994): with s = ceil(log2 d) and m = ceil(2^(31+s) / d) (m < 2^32),
// (n * m) >> (31 + s) equals floor(n / d) for every n < 2^31, because m * d - 2^(31+s) < d <= 2^s.
struct FastDiv {
	uint32_t d, m, s;
};

inline FastDiv MakeFastDiv(uint32_t d)
{
	FastDiv f;
	f.d = d;
	f.s = 0;
	while ((1ull << f.s) < d) { ++f.s; }
	f.m = static_cast<uint32_t>(((1ull << (31 + f.s)) + d - 1) / d);
	return f;
}

__host__ __device__ __forceinline__ uint32_t FastDivide(uint32_t n, const FastDiv& f)
{
	return static_cast<uint32_t>((static_cast<unsigned long long>(n) * f.m) >> (31 + f.s));
}

// Geometry of one chunk: B frames of H x W pixels; global pixel index g = f * N + y * W + x (fits in 31 bits).
struct Geometry {
	int H, W, B;
	int words;  // 32-bit words per row of the root bitmask
	long long N;
	long long P;  // B * N
	FastDiv divN, divW;
};

// Device workspace of one chunk. Dense arrays have P entries, lists have their stated capacities.
struct Workspace {
	Geometry g;
	// dense
	const uint16_t* img;  // the chunk's frames (device)
	uint8_t* code;
	uint32_t* w1;         // W1 in 2^-16 units, valid on domain pixels only (there 0 < W1 < 2^32)
	uint32_t* par;        // union-find parent, then component id tag at roots; once the groups are scattered, the
	                      // parent-chain minimum of W1 of each pixel a global-memory flood pushes (its exactness check)
	uint32_t* lab;        // region id + 1 on labelled domain pixels
	uint32_t* rootmask;   // [B][H][words] bit set at root seeds
	uint32_t* rowcnt;     // [B*H + 1] root seeds per row, scanned in place to row offsets
	// lists
	uint32_t* dom;   uint32_t capDom;
	uint32_t* seeds; uint32_t capSeed;
	// components
	uint32_t capComp;
	uint32_t* compRoot; uint32_t* compSize; uint32_t* compNRoot; uint32_t* compNSeed; uint32_t* compRegion;
	uint32_t* multi;      // ids of multi-region components (groups)
	uint32_t* gOff; uint32_t* gSeedOff; uint32_t* gRegOff;  // exclusive scans over groups
	uint32_t* gCurPix; uint32_t* gCurSeed; uint32_t* gCurReg;
	uint32_t* gPix;  uint32_t* gSeed; uint32_t* gReg;       // per-group pixel, seed and region lists
	double* heapKey; uint32_t* heapPix;                     // per-group heaps (capacity = group size)
	// regions
	uint32_t capRegion;
	uint32_t* regCount; unsigned long long* regSumVJ; unsigned long long* regSumVI; unsigned long long* regSumV;
	uint32_t* regFrame;   // frame (within the chunk) of each region
	uint32_t* regCand;    // exclusive scan of (surf > 4) over regions
	// fusion scratch, indexed by region id
	double* fuMaxWN; double* fuMinP; double* fuMaxP; uint32_t* fuMaxPos; uint32_t* fuWNPos; uint32_t* fuNeighbour;
	uint32_t* fuBecome; uint8_t* fuLocked;
	// per frame [B + 1]: domain pixels and seeds (counted by the detection kernel), 1 where the frame is flooded again
	// frame-wide (its per-component flood failed the exactness check)
	uint32_t* frameDom; uint32_t* frameSeeds; uint32_t* frameRoute;
	// per frame [B + 1]: nonzero where a boundary pair failed the first exactness test (then the frame's rank-test slot
	// + 1); the failing pairs (frame, parent-chain minimum, W1 of the other-label neighbour z, W1 of z's highest
	// domain neighbour); the pairs ordered by slot, with [kRankSlots + 1] slot offsets; two pixel counts per pair
	uint32_t* frameSuspect;
	uint4* suspect; uint32_t capSuspect;
	uint32_t* rankOrder; uint32_t* rankSlotOff; uint32_t* rankCount;
	// per frame [B + 1]: nonzero where the frame failed the rank test (then its re-flood slot + 1); per slot and list
	// (0: the W1 values of its domain pixels, 1: of the pixels its frame-wide flood pops): the values as gathered and
	// grouped by value bucket ([kRefloodSlots][2][kRefloodCap]), the bucket offsets ([kRefloodSlots][2][buckets + 1]);
	// per slot [8]: the two counts, the frame + 1, unused, and per list the lowest value and the bucket shift; per slot
	// and pixel of the frame: the estimated frame-wide pop position and its upper bound, then the global re-flood's
	// element value and chain minimum ([kRefloodSlots][N][kRfWords]); the
	// multi-label groups of the slotted frames ([capComp])
	uint32_t* frameReflood;
	uint32_t* rfVals; uint32_t* rfGrp; uint32_t* rfOff; uint32_t* rfInfo; uint32_t* rfPix; uint32_t* rfGroups;
	uint32_t* frameRegBase; uint32_t* frameCandBase; uint32_t* frameKeep; uint32_t* frameOutBase;
	// candidates / rows
	uint32_t capRows;
	uint32_t* candRegion;  // region of each kept candidate, ordered by (frame, label)
	uint32_t* candFrame;
	struct Cand* cand;     // fit inputs built from the regions
	double* rows;          // [capRows][18], unsorted fit results
	double* sortedRows;    // [capRows][18], per-frame (Y, X) order with Id/Plane/Index
	uint32_t* sortIdx;     // scratch for the per-frame sort
	double* sortKey;
	uint8_t* fitFlag;      // FP32 fits that need an FP64 re-run
	// scan scratch
	uint32_t* scanBlock;   // block sums
	Counters* cnt;
};

}  // namespace ptb
