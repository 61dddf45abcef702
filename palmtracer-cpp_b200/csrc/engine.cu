// Host side of the localization engine: device workspace, the per-chunk kernel chain and the four reference
// operations (Localization, Fitting, Wavelett, AutoThreshold) over host or device buffers.
//
// A call processes its stack in chunks of B frames sized from a device-memory budget. Every list in the workspace
// is sized for the worst case of its chunk (all pixels in the domain, every other pixel a component), so no
// capacity can overflow; the budget only bounds B.
#include "engine.h"

#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <iostream>
#include <mutex>
#include <numeric>
#include <thread>
#include <vector>

namespace ptb {

bool LaunchDetect(const Workspace& ws, double thr, cudaStream_t st);
bool LaunchPlane(const uint16_t* img, double* out, int H, int W, int B, int level, cudaStream_t st);
bool LaunchSegment(const Workspace& ws, double ratio, int strict, uint32_t maxPoints, cudaStream_t st);
bool LaunchBuildCandidates(const Workspace& ws, cudaStream_t st);
bool LaunchSortFrames(const Workspace& ws, double* out, unsigned long long* rowBase, bool offsetOut, unsigned long long planeBase,
                      cudaStream_t st);
bool LaunchFit(const uint16_t* img, int H, int W, long long N, const Cand* cands, const uint32_t* nptr, uint32_t nconst,
               uint32_t cap, const FitParams& fp, double* rows, uint8_t* flags, int precision, cudaStream_t st);
bool LaunchAstigEstimate(const double* dIn, double* dOut, uint64_t n, double pixelSize, const double* model, double zMax, cudaStream_t st);
bool TrackDevice(const double* dIn, uint64_t* dOut, uint64_t nPoints, double maxDistance, cudaStream_t st);

// ---- error plumbing -------------------------------------------------------------------------------------------
namespace {
thread_local std::string g_lastError;
std::atomic<uint64_t> g_launches{0};
}  // namespace

void SetError(const std::string& msg)
{
	if (g_lastError.empty()) { g_lastError = msg; }
}
const std::string& LastError() { return g_lastError; }
void ClearError() { g_lastError.clear(); }
void CountLaunch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
uint64_t LaunchCount() { return g_launches.load(std::memory_order_relaxed); }

bool CheckCuda(cudaError_t e, const char* what, const char* file, int line)
{
	if (e == cudaSuccess) { return true; }
	SetError(std::string(what) + ": " + cudaGetErrorString(e) + " (" + file + ":" + std::to_string(line) + ")");
	return false;
}

// ---- fit parameters ------------------------------------------------------------------------------------------
bool ParseFitParams(uint64_t fit, const double* fp, FitParams& out, std::vector<double>& splineHost)
{
	out = FitParams{};
	out.mode = (fit >= 1 && fit <= 8) ? static_cast<int>(fit) : kNone;
	out.sigmaX = 1.0;
	out.sigmaY = 2.0;
	out.theta = 0.0;
	if (out.mode == kNone) { return true; }
	if (fp == nullptr) {
		SetError("fit_params is null");
		return false;
	}
	if (!(fp[0] >= 1.0) || !std::isfinite(fp[0])) {
		SetError("fit_params[0] (ROI size) must be >= 1");
		return false;
	}
	int roi = static_cast<int>(static_cast<size_t>(fp[0]));
	out.roiParam = fp[0];
	if (out.mode >= kMleGauss) {
		MleParams& m = out.mle;
		m = MleParams{};
		m.model = out.mode;
		if (out.mode == kMleGauss) {
			m.sigma0 = fp[1]; m.offset = fp[2]; m.gain = fp[3]; m.maxIter = static_cast<int>(fp[4]); m.crlbMax = fp[5];
		}
		else if (out.mode == kMleAstig) {
			m.pixelSize = fp[1];
			for (int i = 0; i < 10; ++i) { m.astig[i] = fp[2 + i]; }
			m.offset = fp[12]; m.gain = fp[13]; m.maxIter = static_cast<int>(fp[14]); m.zMin = fp[15]; m.zMax = fp[16];
			m.crlbMax = fp[17];
		}
		else {
			m.sx = static_cast<int>(fp[1]); m.sy = static_cast<int>(fp[2]); m.sz = static_cast<int>(fp[3]); m.dz = fp[4];
			m.offset = fp[5]; m.gain = fp[6]; m.maxIter = static_cast<int>(fp[7]); m.crlbMax = fp[8];
			out.sx = m.sx; out.sy = m.sy; out.sz = m.sz;
			out.splineSize = static_cast<long long>(m.sx) * m.sy * m.sz;
			if (m.sx <= 0 || m.sy <= 0 || m.sz <= 0) { SetError("spline dimensions must be positive"); return false; }
			splineHost.assign(fp + 9, fp + 9 + static_cast<size_t>(out.splineSize) * 64);
		}
		if (roi % 2 == 0) { roi--; }
		m.roi = roi;
		m.half = roi / 2;
		m.n = roi * roi;
		if (!(m.gain > 0) || m.maxIter < 0 || roi > 15) {
			SetError("MLE fit parameters: gain must be > 0, maxIter >= 0 and the ROI at most 15 pixels");
			return false;
		}
		if (out.mode == kMleSpline && (m.sx < roi + 5 || m.sy < roi + 5)) {
			SetError("spline table must be at least ROI + 5 cells wide in x and y");
			return false;
		}
		out.roi = roi; out.half = roi / 2; out.n = roi * roi; out.nParams = 5;
		return true;
	}
	if (out.mode == kSplineEmccd) {
		// [roi, sx, sy, sz, deltaZ, coefficients SoA [64][sz][sy][sx]] (SplineFit.cpp:36-50)
		out.sx = static_cast<int>(static_cast<size_t>(fp[1]));
		out.sy = static_cast<int>(static_cast<size_t>(fp[2]));
		out.sz = static_cast<int>(static_cast<size_t>(fp[3]));
		out.deltaZ = fp[4];
		if (out.sx <= 0 || out.sy <= 0 || out.sz <= 0) {
			SetError("spline dimensions must be positive");
			return false;
		}
		out.splineSize = static_cast<long long>(out.sx) * out.sy * out.sz;
		const size_t ncoef = static_cast<size_t>(out.splineSize) * 64;
		splineHost.assign(fp + 5, fp + 5 + ncoef);
		const double centre = splineHost[(32 * static_cast<size_t>(out.splineSize)) + (out.sz / 2 * static_cast<size_t>(out.sx) * out.sy) +
		                                 (out.sy / 2 * static_cast<size_t>(out.sx)) + (out.sx / 2)];
		out.intensityRatio = std::abs(centre) < 2.220446049250313e-16 ? 1.0 : 4.0 / centre;
		out.offsetXY = static_cast<long long>(std::floor((static_cast<double>(out.sx) + 1.0 - static_cast<double>(roi)) / 2));
		out.initZ = static_cast<double>(out.sz) / 2.0;
		out.nParams = 5;
	}
	else {
		out.sigmaX = fp[1];
		out.sigmaY = fp[2];
		out.theta = fp[3];
		out.nParams = out.mode == kG2Fixed ? 4 : out.mode == kG2Sigma ? 5 : out.mode == kG3Fixed ? 6 : 7;
	}
	if (roi % 2 == 0) { roi--; }
	out.roi = roi;
	out.half = roi / 2;
	out.n = roi * roi;
	return true;
}

size_t FitParamCount(uint64_t fit, const double* fp)
{
	if (fp == nullptr) { return 0; }
	auto cells = [](double a, double b, double c) {
		return static_cast<size_t>(std::max(0.0, a)) * static_cast<size_t>(std::max(0.0, b)) * static_cast<size_t>(std::max(0.0, c));
	};
	switch (fit) {
		case kG2Fixed: case kG2Sigma: case kG3Fixed: case kG3Theta: return 4;
		case kSplineEmccd: return 5 + 64 * cells(fp[1], fp[2], fp[3]);
		case kMleGauss: return 6;
		case kMleAstig: return 18;
		case kMleSpline: return 9 + 64 * cells(fp[1], fp[2], fp[3]);
		default: return 0;
	}
}

// ---- workspace ------------------------------------------------------------------------------------------------
namespace {

size_t Align(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

// Words of the per-chunk frame arrays zeroed before each chunk: five [B + 1] arrays.
size_t FrameWords(int B) { return 5 * (static_cast<size_t>(B) + 1); }

uint32_t IndepBound(int H, int W) { return static_cast<uint32_t>(((H + 1) / 2)) * static_cast<uint32_t>(((W + 1) / 2)); }

}  // namespace

// Host memcpy over several threads (pageable buffers go through pinned staging; one thread copies about 10 GB/s).
void ParallelCopy(void* dst, const void* src, size_t bytes)
{
	const size_t piece = 32ull << 20;
	const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
	const unsigned n = static_cast<unsigned>(std::min<size_t>(hw, (bytes + piece - 1) / piece));
	if (n <= 1) {
		std::memcpy(dst, src, bytes);
		return;
	}
	std::vector<std::thread> th;
	const size_t each = (bytes / n + 63) & ~static_cast<size_t>(63);
	for (unsigned i = 0; i < n; ++i) {
		const size_t a = std::min(bytes, each * i), b = std::min(bytes, each * (i + 1));
		if (b > a) { th.emplace_back([=] { std::memcpy(static_cast<char*>(dst) + a, static_cast<const char*>(src) + a, b - a); }); }
	}
	for (auto& t : th) { t.join(); }
}

// True for host memory that is neither page-locked nor registered with CUDA.
bool Pageable(const void* p)
{
	cudaPointerAttributes a{};
	if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
		cudaGetLastError();
		return true;
	}
	return a.type == cudaMemoryTypeUnregistered;
}

// Bytes of workspace for B frames of H x W with `rowsCap` fit rows.
static size_t PlanWorkspace(Workspace& ws, int H, int W, int B, uint32_t rowsCap, char* base)
{
	Geometry g;
	g.H = H;
	g.W = W;
	g.B = B;
	g.words = (W + 31) / 32;
	g.N = static_cast<long long>(H) * W;
	g.P = g.N * B;
	g.divN = MakeFastDiv(static_cast<uint32_t>(g.N));
	g.divW = MakeFastDiv(static_cast<uint32_t>(W));
	ws.g = g;
	const size_t P = static_cast<size_t>(g.P);
	const uint32_t capComp = IndepBound(H, W) * static_cast<uint32_t>(B) + 1;
	ws.capDom = static_cast<uint32_t>(P);
	ws.capSeed = static_cast<uint32_t>(P);
	ws.capComp = capComp;
	ws.capRegion = capComp;
	ws.capRows = std::max<uint32_t>(1, std::min<uint32_t>(rowsCap, capComp));
	size_t off = 0;
	auto take = [&](auto*& ptr, size_t count) {
		using T = std::remove_pointer_t<std::remove_reference_t<decltype(ptr)>>;
		const size_t bytes = Align(std::max<size_t>(count, 1) * sizeof(T));
		if (base) { ptr = reinterpret_cast<T*>(base + off); }
		off += bytes;
	};
	const size_t rows = static_cast<size_t>(g.B) * g.H;
	take(ws.code, P);
	take(ws.w1, P);
	take(ws.par, P);
	take(ws.lab, P);
	take(ws.rootmask, rows * g.words);
	take(ws.rowcnt, rows + 1);
	take(ws.dom, P);
	take(ws.seeds, P);
	take(ws.compRoot, capComp);
	take(ws.compSize, capComp);
	take(ws.compNRoot, capComp);
	take(ws.compNSeed, capComp);
	take(ws.compRegion, capComp);
	take(ws.multi, capComp);
	take(ws.gOff, capComp + 1);
	take(ws.gSeedOff, capComp + 1);
	take(ws.gRegOff, capComp + 1);
	take(ws.gCurPix, capComp + 1);
	take(ws.gCurSeed, capComp + 1);
	take(ws.gCurReg, capComp + 1);
	take(ws.gPix, P);
	take(ws.gSeed, P);
	take(ws.gReg, capComp);
	take(ws.heapKey, P);
	take(ws.heapPix, P);
	take(ws.regCount, capComp);
	take(ws.regSumVJ, capComp);
	take(ws.regSumVI, capComp);
	take(ws.regSumV, capComp);
	take(ws.regFrame, capComp);
	take(ws.regCand, capComp + 1);
	take(ws.fuMaxWN, capComp);
	take(ws.fuMinP, capComp);
	take(ws.fuMaxP, capComp);
	take(ws.fuMaxPos, capComp);
	take(ws.fuWNPos, capComp);
	take(ws.fuNeighbour, capComp);
	take(ws.fuBecome, capComp);
	take(ws.fuLocked, capComp);
	// frameDom, frameSeeds, frameRoute, frameSuspect and frameReflood (zeroed together for each chunk)
	take(ws.frameDom, FrameWords(B));
	if (base) {
		ws.frameSeeds = ws.frameDom + B + 1;
		ws.frameRoute = ws.frameSeeds + B + 1;
		ws.frameSuspect = ws.frameRoute + B + 1;
		ws.frameReflood = ws.frameSuspect + B + 1;
	}
	take(ws.rfVals, static_cast<size_t>(kRefloodSlots) * 2 * kRefloodCap);
	take(ws.rfGrp, static_cast<size_t>(kRefloodSlots) * 2 * kRefloodCap);
	take(ws.rfOff, static_cast<size_t>(kRefloodSlots) * 2 * (kRefloodBuckets + 1));
	take(ws.rfInfo, static_cast<size_t>(kRefloodSlots) * 8);
	take(ws.rfPix, static_cast<size_t>(kRefloodSlots) * static_cast<size_t>(g.N) * kRfWords);
	take(ws.rfGroups, capComp);
	take(ws.suspect, kSuspectCap);
	take(ws.rankOrder, kSuspectCap);
	take(ws.rankSlotOff, kRankSlots + 1);
	take(ws.rankCount, 2 * kSuspectCap);
	ws.capSuspect = kSuspectCap;
	take(ws.frameRegBase, static_cast<size_t>(B) + 1);
	take(ws.frameCandBase, static_cast<size_t>(B) + 1);
	take(ws.frameKeep, static_cast<size_t>(B) + 1);
	take(ws.frameOutBase, static_cast<size_t>(B) + 1);
	take(ws.candRegion, ws.capRows);
	take(ws.candFrame, ws.capRows);
	take(ws.cand, ws.capRows);
	take(ws.rows, static_cast<size_t>(ws.capRows) * kCols);
	take(ws.sortedRows, static_cast<size_t>(ws.capRows) * kCols);
	take(ws.sortIdx, static_cast<size_t>(ws.capRows) * 2);
	take(ws.sortKey, static_cast<size_t>(ws.capRows) * 4);
	take(ws.fitFlag, ws.capRows);
	take(ws.scanBlock, P / 4096 + 64);
	take(ws.cnt, 1);
	return off;
}

Engine::Engine() = default;

Engine::~Engine()
{
	for (auto& list : graphs_) {
		for (auto& g : list) { cudaGraphExecDestroy(g.exec); }
	}
	if (pool_) { cudaFree(pool_); }
	if (img_) { cudaFree(img_); }
	if (hostStage_) { cudaFreeHost(hostStage_); }
	for (void* h : hostOut_) {
		if (h) { cudaFreeHost(h); }
	}
	if (spline_) { cudaFree(spline_); }
	if (fallbacks_) { cudaFree(fallbacks_); }
	if (evalDev_) { cudaFree(evalDev_); }
	if (rowBase_) { cudaFree(rowBase_); }
	if (hostCnt_) { cudaFreeHost(hostCnt_); }
	if (copy_) { cudaStreamDestroy(copy_); }
	if (copyOut_) { cudaStreamDestroy(copyOut_); }
	if (pool1_) { cudaFree(pool1_); }
	if (stream1_) { cudaStreamDestroy(stream1_); }
	if (stream_) { cudaStreamDestroy(stream_); }
}

bool Engine::Init()
{
	if (stream_) { return true; }
	if (!PTB_CUDA(cudaGetDevice(&device_))) { return false; }
	if (const char* env = std::getenv("PTB_GRAPHS")) { useGraphs_ = std::atoi(env) != 0; }
	if (!PTB_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking))) { return false; }
	if (!PTB_CUDA(cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking))) { return false; }
	if (!PTB_CUDA(cudaStreamCreateWithFlags(&copyOut_, cudaStreamNonBlocking))) { return false; }
	if (!PTB_CUDA(cudaStreamCreateWithFlags(&stream1_, cudaStreamNonBlocking))) { return false; }
	for (auto& e : sortDone_) {
		if (!PTB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming))) { return false; }
	}
	if (!PTB_CUDA(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming))) { return false; }
	if (!PTB_CUDA(cudaMallocHost(&hostCnt_, 2 * sizeof(Counters)))) { return false; }
	if (!PTB_CUDA(cudaMalloc(&rowBase_, sizeof(unsigned long long)))) { return false; }
	for (cudaEvent_t* e : {&h2d_[0], &h2d_[1], &h2d_[2], &imgFree_[0], &imgFree_[1], &imgFree_[2], &done_[0], &done_[1], &d2h_[0], &d2h_[1],
	                       &outEv_[0], &outEv_[1]}) {
		if (!PTB_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming))) { return false; }
	}
	for (auto& e : ev_) {
		if (!PTB_CUDA(cudaEventCreate(&e))) { return false; }
	}
	for (auto& e : mleEv_) {
		if (!PTB_CUDA(cudaEventCreate(&e))) { return false; }
	}
	size_t freeB = 0, totalB = 0;
	if (!PTB_CUDA(cudaMemGetInfo(&freeB, &totalB))) { return false; }
	// default budget: a quarter of free memory, at most 48 GiB (leaves room for callers' own buffers); on a B200 about
	// 280 frames of 1024 x 1024 per chunk slot, which halves the chunks (and their serial tails) of 24 GiB
	budget_ = std::min<size_t>(freeB / 4, 48ull << 30);
	if (const char* env = std::getenv("PTB_WORKSPACE_MB")) { budget_ = static_cast<size_t>(std::atoll(env)) << 20; }
	if (fixedBudget_) { budget_ = fixedBudget_; }
	return true;
}

bool Engine::Reserve(int H, int W, int B, uint32_t rowsCap, int slots)
{
	Workspace probe{};
	const size_t need = PlanWorkspace(probe, H, W, B, rowsCap, nullptr);
	if (need > poolBytes_) {
		if (pool_) { cudaFree(pool_); pool_ = nullptr; poolBytes_ = 0; }
		if (!PTB_CUDA(cudaMalloc(&pool_, need))) { return false; }
		poolBytes_ = need;
	}
	PlanWorkspace(ws_, H, W, B, rowsCap, static_cast<char*>(pool_));
	if (slots > 1) {
		if (need > pool1Bytes_) {
			if (pool1_) { cudaFree(pool1_); pool1_ = nullptr; pool1Bytes_ = 0; }
			if (!PTB_CUDA(cudaMalloc(&pool1_, need))) { return false; }
			pool1Bytes_ = need;
		}
		PlanWorkspace(ws1_, H, W, B, rowsCap, static_cast<char*>(pool1_));
	}
	return true;
}

bool Engine::ReserveImage(size_t bytes)
{
	if (bytes <= imgBytes_) { return true; }
	if (img_) { cudaFree(img_); img_ = nullptr; imgBytes_ = 0; }
	if (!PTB_CUDA(cudaMalloc(&img_, bytes))) { return false; }
	imgBytes_ = bytes;
	return true;
}

size_t Engine::EstimateBytes(uint64_t height, uint64_t width, uint64_t planes, uint64_t outputSize) const
{
	if (planes == 0 || height == 0 || width == 0) { return 0; }
	const int H = static_cast<int>(height), W = static_cast<int>(width);
	const uint32_t maxPoints = static_cast<uint32_t>(std::min<uint64_t>((outputSize / kCols) / planes, 0xffffffffu));
	int B = 1, slots = 1;
	ChunkPlan(H, W, planes, maxPoints, B, slots);
	const uint32_t rowsCap = static_cast<uint32_t>(std::min<uint64_t>(static_cast<uint64_t>(B) * maxPoints, 0xffffffffu));
	Workspace probe{};
	const size_t ws = PlanWorkspace(probe, H, W, B, rowsCap, nullptr);
	const size_t img = 2ull * static_cast<size_t>(H) * W * B * sizeof(uint16_t);
	return slots * ws + img;
}

int Engine::ChunkFrames(int H, int W, uint64_t planes, uint32_t maxPoints, size_t budget) const
{
	const long long N = static_cast<long long>(H) * W;
	// bytes per frame: ~40 B per pixel of dense lists plus ~100 B per independent-set slot plus fit rows
	const double perFrame = 48.0 * N + 100.0 * IndepBound(H, W) +
	                        std::min<double>(maxPoints, IndepBound(H, W)) * 360.0 + 2.0 * N;
	long long B = static_cast<long long>(static_cast<double>(budget) / perFrame);
	B = std::max<long long>(1, std::min<long long>(B, static_cast<long long>(planes)));
	// global pixel indices of a chunk stay below 2^31 (the top bit tags component ids)
	B = std::min<long long>(B, std::max<long long>(1, ((1ll << 31) - 1) / std::max<long long>(N, 1)));
	// the per-frame kernels (detection, wavelet planes, tile components) take the frame from grid.z
	B = std::min<long long>(B, 65535);
	return static_cast<int>(B);
}

// One chunk when the whole stack fits the budget; otherwise two chunk slots with half the budget each, so that two
// chunks are in flight on two compute streams.
void Engine::ChunkPlan(int H, int W, uint64_t planes, uint32_t maxPoints, int& B, int& slots) const
{
	B = ChunkFrames(H, W, planes, maxPoints, budget_);
	slots = 1;
	static const int maxSlots = [] { const char* e = std::getenv("PTB_CHUNK_SLOTS"); return e ? std::atoi(e) : 2; }();
	if (static_cast<uint64_t>(B) < planes && maxSlots >= 2) {
		B = ChunkFrames(H, W, planes, maxPoints, budget_ / 2);
		slots = 2;
	}
}

// Size class of a chunk for the fit autotuner: the bit length of its pixel count. Which ROI mapping is faster depends
// on how many ROIs one launch fits (a warp per ROI finishes a small batch sooner; a thread per ROI has the higher
// throughput once the batch fills the GPU many times over), and the candidate count grows with the pixel count.
static int SizeClass(int B, int H, int W)
{
	uint64_t p = static_cast<uint64_t>(B) * static_cast<uint64_t>(H) * static_cast<uint64_t>(W);
	int c = 0;
	while (p) { ++c; p >>= 1; }
	return c;
}

static int TuneKey(const FitParams& fp, int sizeClass) { return (fp.mode * 64 + fp.roi) * 64 + sizeClass; }

// Key of a chunk's launch chain: every value that the captured launches take by value (workspace plan, image
// pointer, threshold, segmentation settings, fit configuration). Two chunks with equal keys launch identical kernels
// with identical arguments, so a graph captured for one replays the other.
static std::vector<uint64_t> ChainKey(int slot, const Workspace& ws, const uint16_t* dImg, double thr, double ratio,
                                      int strict, uint32_t maxPoints, uint32_t rowsCap, int precision, const FitParams& f)
{
	std::vector<uint64_t> k;
	k.reserve(64);
	auto u = [&](uint64_t v) { k.push_back(v); };
	auto d = [&](double v) { uint64_t b; std::memcpy(&b, &v, sizeof b); k.push_back(b); };
	auto p = [&](const void* v) { k.push_back(reinterpret_cast<uintptr_t>(v)); };
	u(static_cast<uint64_t>(slot)); p(ws.code); p(dImg);
	u(static_cast<uint64_t>(ws.g.H)); u(static_cast<uint64_t>(ws.g.W)); u(static_cast<uint64_t>(ws.g.B)); u(rowsCap);
	d(thr); d(ratio); u(static_cast<uint64_t>(strict)); u(maxPoints); u(static_cast<uint64_t>(precision));
	u(static_cast<uint64_t>(f.mode)); u(static_cast<uint64_t>(f.roi)); u(static_cast<uint64_t>(f.half));
	u(static_cast<uint64_t>(f.n)); u(static_cast<uint64_t>(f.nParams)); d(f.sigmaX); d(f.sigmaY); d(f.theta);
	u(static_cast<uint64_t>(f.sx)); u(static_cast<uint64_t>(f.sy)); u(static_cast<uint64_t>(f.sz));
	u(static_cast<uint64_t>(f.splineSize)); u(static_cast<uint64_t>(f.offsetXY)); d(f.roiParam); d(f.initZ); d(f.deltaZ);
	d(f.intensityRatio); p(f.coeffs); u(static_cast<uint64_t>(f.lanes)); p(f.marks);
	const MleParams& m = f.mle;
	u(static_cast<uint64_t>(m.model)); u(static_cast<uint64_t>(m.roi)); u(static_cast<uint64_t>(m.half));
	u(static_cast<uint64_t>(m.n)); u(static_cast<uint64_t>(m.maxIter)); u(static_cast<uint64_t>(m.chunk)); d(m.sigma0);
	d(m.offset); d(m.gain); d(m.crlbMax);
	d(m.pixelSize); d(m.zMin); d(m.zMax);
	for (double a : m.astig) { d(a); }
	u(static_cast<uint64_t>(m.sx)); u(static_cast<uint64_t>(m.sy)); u(static_cast<uint64_t>(m.sz)); d(m.dz);
	p(m.table); p(m.table64); p(m.fallbacks); p(m.queue); p(m.evals);
	return k;
}

Engine::GraphEntry* Engine::FindGraph(int slot, const std::vector<uint64_t>& key)
{
	for (auto& e : graphs_[slot]) {
		if (e.key == key) {
			e.lastUse = ++graphClock_;
			return &e;
		}
	}
	return nullptr;
}

// Captures the compute part of a chunk (launch) on the slot's stream into a graph and keeps its executable (evicting
// the least recently used of kGraphsPerSlot). Returns false, with no error recorded, when the capture or the
// instantiation fails; the caller then launches directly.
Engine::GraphEntry* Engine::CaptureGraph(int slot, std::vector<uint64_t> key, const std::function<bool()>& launch)
{
	cudaStream_t st = St(slot);
	const std::string before = LastError();
	cudaGraph_t graph = nullptr;
	cudaGraphExec_t exec = nullptr;
	const uint64_t l0 = LaunchCount();
	bool ok = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
	if (ok) {
		const bool launched = launch();
		ok = cudaStreamEndCapture(st, &graph) == cudaSuccess && launched;
	}
	const uint64_t launches = LaunchCount() - l0;
	ok = ok && cudaGraphInstantiateWithFlags(&exec, graph, 0) == cudaSuccess;
	if (graph) { cudaGraphDestroy(graph); }
	if (!ok) {
		// leave no trace of the failed capture: the chunk is launched directly instead
		if (exec) { cudaGraphExecDestroy(exec); }
		cudaGetLastError();
		ClearError();
		if (!before.empty()) { SetError(before); }
		graphsOff_ = true;
		return nullptr;
	}
	auto& list = graphs_[slot];
	if (list.size() >= kGraphsPerSlot) {
		auto lru = std::min_element(list.begin(), list.end(), [](const GraphEntry& a, const GraphEntry& b) { return a.lastUse < b.lastUse; });
		cudaGraphExecDestroy(lru->exec);
		list.erase(lru);
	}
	// the captured launches were counted while recording; the first replay is therefore not counted again
	list.push_back(GraphEntry{std::move(key), exec, launches, ++graphClock_, true});
	return &list.back();
}

// Runs detection -> segmentation -> fits -> ordering for B frames whose pixels are at dImg (device). The chunk's
// rows go to dOut (device) numbered from Id idBase + 1 and Plane planeBase + 1; returns the row count or -1.
// The compute part (counters reset through the fits) is replayed from a CUDA graph when an earlier chunk had the same
// launch chain (the second occurrence of a chain captures it); the ordering step, which follows the other slot's
// ordering, is launched directly.
bool Engine::EnqueueChunk(int slot, const uint16_t* dImg, int H, int W, int B, double thr, double ratio, uint32_t maxPoints,
                          const FitParams& fp, double* dOut, bool offsetOut, unsigned long long planeBase, bool afterOther)
{
	Workspace& ws = Ws(slot);
	ws.img = dImg;
	cudaStream_t st = St(slot);
	const bool prof = profiling_ != 0;
	segCounts_[0] += static_cast<uint64_t>(B);
	uint64_t l0 = LaunchCount();
	auto mark = [&](int k) {
		if (prof) {
			cudaEventRecord(ev_[k], st);
			if (k > 0) { pendLaunches_[k - 1] = LaunchCount() - l0; l0 = LaunchCount(); }
		}
	};
	FitParams fpr = fp;
	const bool hooked = fitHook_ && fpr.mode >= kMleGauss;  // the fit runs in the hook's stage, outside this chain
	if (fpr.mode >= kMleGauss && !hooked) {
		if (fpr.lanes == 0) { TunedMapping(fpr, SizeClass(B, H, W)); }
		fpr.mle.queue = ws.cnt->queue;  // this slot's work-queue counters
	}
	const bool tune = !hooked && fpr.mode >= kMleGauss && fpr.lanes == 0;  // first chunk of this class: time the mappings
	pendMleProf_ = prof && fpr.mode >= kMleGauss && !hooked;
	bool ok = true;
	if (pendMleProf_) {
		if (!evalDev_) { ok = ok && PTB_CUDA(cudaMalloc(&evalDev_, 3 * sizeof(unsigned long long))); }
		ok = ok && PTB_CUDA(cudaMemsetAsync(evalDev_, 0, 3 * sizeof(unsigned long long), st));
		fpr.marks = mleEv_;
		fpr.mle.evals = evalDev_;
	}
	const uint32_t rowsCap = ws.capRows;
	auto segmentAndDetect = [&]() {
		bool k = PTB_CUDA(cudaMemsetAsync(ws.cnt, 0, sizeof(Counters), st));
		k = k && PTB_CUDA(cudaMemsetAsync(ws.rootmask, 0, sizeof(uint32_t) * static_cast<size_t>(B) * H * ws.g.words, st));
		k = k && PTB_CUDA(cudaMemsetAsync(ws.frameDom, 0, sizeof(uint32_t) * FrameWords(B), st));
		mark(0);
		k = k && LaunchDetect(ws, thr, st);
		mark(1);
		k = k && LaunchSegment(ws, ratio, strict_, maxPoints, st);
		k = k && LaunchBuildCandidates(ws, st);
		mark(2);
		return k;
	};
	auto fit = [&]() {
		if (hooked) { return true; }  // after the chain, below
		return LaunchFit(dImg, H, W, ws.g.N, ws.cand, &ws.cnt->nfit, 0, ws.capRows, fpr, ws.rows, ws.fitFlag, precision_, st);
	};
	bool direct = true;
	if (ok && !prof && !tune && !graphsOff_ && useGraphs_) {
		std::vector<uint64_t> key = ChainKey(slot, ws, dImg, thr, ratio, strict_, maxPoints, rowsCap, precision_, fpr);
		key.push_back(hooked ? 1u : 0u);
		GraphEntry* g = FindGraph(slot, key);
		if (!g) {
			auto seen = std::find(seen_[slot].begin(), seen_[slot].end(), key);
			if (seen != seen_[slot].end()) {
				seen_[slot].erase(seen);
				g = CaptureGraph(slot, std::move(key), [&]() { return segmentAndDetect() && fit(); });
			}
			else {
				if (seen_[slot].size() >= kGraphsPerSlot) { seen_[slot].erase(seen_[slot].begin()); }
				seen_[slot].push_back(std::move(key));
			}
		}
		if (g) {
			ok = PTB_CUDA(cudaGraphLaunch(g->exec, st));
			if (!g->fresh) { CountLaunch(g->launches); }
			++graphCounts_[g->fresh ? 0 : 1];
			g->fresh = false;
			direct = false;
		}
	}
	if (direct) {
		++graphCounts_[2];
		ok = ok && segmentAndDetect();
		if (ok && tune) { ok = Autotune(fpr, dImg, H, W, slot, SizeClass(B, H, W)); }
		ok = ok && fit();
	}
	if (ok && hooked) {
		const FitJob job{st, FitImage{dImg, H, W, ws.g.N}, ws.cand, &ws.cnt->nfit, ws.capRows, ws.rows, fpr};
		ok = fitHook_(job);
	}
	pendLanes_ = fpr.lanes;
	mark(3);
	if (afterOther) { ok = ok && PTB_CUDA(cudaStreamWaitEvent(st, sortDone_[1 - slot], 0)); }
	ok = ok && LaunchSortFrames(ws, dOut, rowBase_, offsetOut, planeBase, st);
	ok = ok && PTB_CUDA(cudaEventRecord(sortDone_[slot], st));
	mark(4);
	ok = ok && PTB_CUDA(cudaMemcpyAsync(hostCnt_ + slot, ws.cnt, sizeof(Counters), cudaMemcpyDeviceToHost, st));
	ok = ok && PTB_CUDA(cudaEventRecord(done_[slot], st));
	return ok;
}

long long Engine::CompleteChunk(int slot, uint32_t* truncatedFrames)
{
	if (!PTB_CUDA(cudaEventSynchronize(done_[slot]))) { return -1; }
	if (profiling_) {
		for (int k = 0; k < 4; ++k) {
			float ms = 0.f;
			cudaEventElapsedTime(&ms, ev_[k], ev_[k + 1]);
			stageMs_[k] += ms;
			stageLaunches_[k] += pendLaunches_[k];
		}
	}
	if (pendMleProf_) {
		for (int k = 0; k < 4; ++k) {
			float ms = 0.f;
			cudaEventElapsedTime(&ms, mleEv_[k], mleEv_[k + 1]);
			stageMs_[5 + k] += ms;
			stageLaunches_[5 + k] += (k == 1 || pendLanes_ == 1) ? 1 : 0;
		}
		unsigned long long ev[3] = {};
		if (!PTB_CUDA(cudaMemcpy(ev, evalDev_, sizeof(ev), cudaMemcpyDeviceToHost))) { return -1; }
		for (int k = 0; k < 3; ++k) { evalTotals_[k] += ev[k]; }
		pendMleProf_ = false;
	}
	const Counters& c = hostCnt_[slot];
	if (c.overflow) {
		SetError("internal capacity overflow");
		return -1;
	}
	if (c.fault) {
		SetError("the detection kernel's wait for its staged input tile ran out");
		return -1;
	}
	segCounts_[1] += c.nroute;
	segCounts_[2] += c.nslots;
	segCounts_[3] += c.nreflood;
	for (int k = 0; k < 7; ++k) { segCounts_[4 + k] += c.routeWhy[k]; }
	if (truncatedFrames) { *truncatedFrames += c.truncated; }
	return c.nfit;
}

// Frame counts of the chunks of a stack of `planes` frames, at most B each. Device input: B frames each, the last one
// shorter. Host input, where the copy-in is the critical path: the stack's end is cut into chunks that shrink by a
// factor of about 0.7 down to about B / 16 frames, so that each chunk computes while the next, smaller one is copied
// in and little compute is left after the final copy-in; the rest is cut into equal chunks of at most B, of which
// the first is split so that compute starts after a copy-in of about B / 8 frames.
static void ChunkSchedule(uint64_t planes, uint64_t B, bool hostInput, std::vector<uint64_t>& count)
{
	count.clear();
	if (!hostInput || planes <= B) {
		for (uint64_t z0 = 0; z0 < planes; z0 += B) { count.push_back(std::min<uint64_t>(B, planes - z0)); }
		return;
	}
	std::vector<uint64_t> back;  // the end, last chunk first
	uint64_t left = planes;
	for (uint64_t t = std::max<uint64_t>(1, B / 16); left > 0 && t < B; t = std::max(t + 1, t * 10 / 7)) {
		back.push_back(std::min(t, left));
		left -= back.back();
	}
	if (left > 0) {
		const uint64_t n = (left + B - 1) / B;
		for (uint64_t k = 0; k < n; ++k) { count.push_back(left / n + (k < left % n ? 1 : 0)); }
		const uint64_t head = std::max<uint64_t>(1, B / 8);
		if (count.front() > head) {
			count.insert(count.begin() + 1, count.front() - head);
			count.front() = head;
		}
	}
	count.insert(count.end(), back.rbegin(), back.rend());
}

// A stack that fits the budget runs as one chunk. A longer one runs as chunks of half the budget on two chunk slots,
// each with its own compute stream and workspace, so that one chunk's serial tail (the last fits, the ordering)
// overlaps the next chunk's detection. With host buffers, the input of chunk k + 1 is copied in on one copy stream and
// the rows of chunk k - 1 are copied out on another while chunk k computes (two staging slots for the frames). Row
// numbering continues across chunks through a device-side row count that each chunk's ordering step advances after
// the previous chunk's, so the host waits for a chunk only to learn how many rows it copies out.
long long Engine::Localize(const uint16_t* input, bool inputOnDevice, double* output, bool outputOnDevice, uint64_t outputSize,
                           uint64_t height, uint64_t width, uint64_t planes, double thr, double ratio, uint64_t fit,
                           const double* fitParams, const PageSource* source)
{
	if (source && (inputOnDevice || outputOnDevice)) {
		SetError("a page source takes host output");
		return -1;
	}
	if (planes == 0 || height == 0 || width == 0) { return 0; }
	const uint64_t perPlane = (outputSize / kCols) / planes;
	if (perPlane == 0) { return 0; }
	if (height > (1u << 30) || width > (1u << 30) || height * width > (1ull << 31) - 1) {
		SetError("frame too large");
		return -1;
	}
	if (!Init()) { return -1; }
	FitParams fp;
	std::vector<double>& spline = splineIn_;
	if (!ParseFitParams(fit, fitParams, fp, spline)) { return -1; }
	if (!UploadSpline(fp, spline)) { return -1; }
	const int H = static_cast<int>(height), W = static_cast<int>(width);
	const uint32_t maxPoints = static_cast<uint32_t>(std::min<uint64_t>(perPlane, 0xffffffffu));
	// pageable host buffers: the frames are copied into pinned staging by several host threads (a page source), and
	// the rows reach the caller's buffer through pinned staging the same way; a copy from or to pageable memory would
	// otherwise go through the driver's single staging buffer and block this thread
	PageSource pageableIn;
	if (!source && !inputOnDevice && !outputOnDevice && Pageable(input)) {
		const size_t frameElems = static_cast<size_t>(H) * W;
		pageableIn = [input, frameElems](uint64_t z0, uint64_t n, uint16_t* dst) {
			ParallelCopy(dst, input + z0 * frameElems, static_cast<size_t>(n) * frameElems * sizeof(uint16_t));
			return true;
		};
		source = &pageableIn;
	}
	const bool stageOut = !outputOnDevice && Pageable(output);
	struct Pending {
		double* dst = nullptr;
		size_t bytes = 0;
	} pending[2];
	// the staged rows of buffer b into the caller's buffer (after their copy from the device)
	auto flushOut = [&](int b) {
		if (!pending[b].dst) { return true; }
		if (!PTB_CUDA(cudaEventSynchronize(outEv_[b]))) { return false; }
		ParallelCopy(pending[b].dst, hostOut_[b], pending[b].bytes);
		pending[b].dst = nullptr;
		return true;
	};
	uint64_t outCopies = 0;
	int B = 1, slots = 1;
	ChunkPlan(H, W, planes, maxPoints, B, slots);
	const uint32_t rowsCap = static_cast<uint32_t>(std::min<uint64_t>(static_cast<uint64_t>(B) * maxPoints, 0xffffffffu));
	if (!Reserve(H, W, B, rowsCap, slots)) { return -1; }
	char* poolOf[2] = {static_cast<char*>(pool_), static_cast<char*>(pool1_)};
	const size_t N = static_cast<size_t>(H) * W;
	std::vector<uint64_t> first, count;
	ChunkSchedule(planes, static_cast<uint64_t>(B), !inputOnDevice, count);
	for (uint64_t k = 0, z0 = 0; k < count.size(); z0 += count[k], ++k) { first.push_back(z0); }
	const uint64_t chunks = first.size();
	const size_t slotBytes = N * B * sizeof(uint16_t);
	// host input: frames go through up to three device staging slots (chunk k in slot k % 3), so that a copy-in waits
	// for the chunk three back, not for the one still computing beside the current one
	const uint64_t imgSlots = std::min<uint64_t>(chunks, 3);
	if (!inputOnDevice && !ReserveImage(imgSlots * slotBytes)) { return -1; }
	if (source && hostStageBytes_ < (chunks > 1 ? 2 : 1) * slotBytes) {
		if (hostStage_) { cudaFreeHost(hostStage_); hostStage_ = nullptr; hostStageBytes_ = 0; }
		if (!PTB_CUDA(cudaMallocHost(&hostStage_, (chunks > 1 ? 2 : 1) * slotBytes))) { return -1; }
		hostStageBytes_ = (chunks > 1 ? 2 : 1) * slotBytes;
	}
	// with two chunk slots, chunk k runs on chunk slot k % 2 (its own stream, workspace, counters and events), with one
	// on slot 0; with host output its ordered rows stay in that workspace (where the chunk's own plan puts them) until
	// copied out
	double* outSlot[2] = {nullptr, nullptr};
	auto chunkSlot = [&](uint64_t k) { return slots > 1 ? static_cast<int>(k & 1) : 0; };
	auto imgSlotOf = [&](uint64_t k) { return static_cast<int>(k % imgSlots); };
	auto imgSlot = [&](int slot) { return static_cast<uint16_t*>(img_) + N * B * slot; };
	auto framesOf = [&](uint64_t k) { return static_cast<int>(count[k]); };
	if (!PTB_CUDA(cudaMemsetAsync(rowBase_, 0, sizeof(unsigned long long), stream_))) { return -1; }
	// the second compute stream starts after everything ordered before this call on the first (the caller's input)
	if (slots > 1 && (!PTB_CUDA(cudaEventRecord(fork_, stream_)) || !PTB_CUDA(cudaStreamWaitEvent(stream1_, fork_, 0)))) {
		return -1;
	}
	// input of chunk k into its staging slot; the slot's previous chunk (k - imgSlots) must have finished reading it
	auto copyIn = [&](uint64_t k) {
		const int slot = imgSlotOf(k);
		const uint16_t* src = source ? nullptr : input + first[k] * N;
		if (source) {
			// the pinned host slot's previous frames (chunk k - 2) must have reached the device before it is refilled
			uint16_t* stage = static_cast<uint16_t*>(hostStage_) + ((k & 1) ? N * B : 0);
			if (k >= 2 && !PTB_CUDA(cudaEventSynchronize(h2d_[imgSlotOf(k - 2)]))) { return false; }
			if (!(*source)(first[k], count[k], stage)) {
				SetError("page source failed");
				return false;
			}
			src = stage;
		}
		if (k >= imgSlots && !PTB_CUDA(cudaStreamWaitEvent(copy_, imgFree_[slot], 0))) { return false; }
		if (!PTB_CUDA(cudaMemcpyAsync(imgSlot(slot), src, N * framesOf(k) * sizeof(uint16_t), cudaMemcpyHostToDevice, copy_))) {
			return false;
		}
		return PTB_CUDA(cudaEventRecord(h2d_[slot], copy_));
	};
	unsigned long long rows = 0;
	uint32_t truncated = 0;
	// waits for chunk k and, for host output, copies its rows out
	auto complete = [&](uint64_t k) {
		const int slot = chunkSlot(k);
		const long long n = CompleteChunk(slot, &truncated);
		if (n < 0) { return false; }
		if (!outputOnDevice && n > 0) {
			const size_t bytes = static_cast<size_t>(n) * kCols * sizeof(double);
			if (stageOut) {
				const int b = static_cast<int>(outCopies++ & 1);
				if (!flushOut(b)) { return false; }
				if (hostOutBytes_[b] < bytes) {
					if (hostOut_[b]) { cudaFreeHost(hostOut_[b]); hostOut_[b] = nullptr; hostOutBytes_[b] = 0; }
					if (!PTB_CUDA(cudaMallocHost(&hostOut_[b], bytes))) { return false; }
					hostOutBytes_[b] = bytes;
				}
				if (!PTB_CUDA(cudaMemcpyAsync(hostOut_[b], outSlot[slot], bytes, cudaMemcpyDeviceToHost, copyOut_)) ||
				    !PTB_CUDA(cudaEventRecord(outEv_[b], copyOut_))) {
					return false;
				}
				pending[b].dst = output + rows * kCols;
				pending[b].bytes = bytes;
			}
			else if (!PTB_CUDA(cudaMemcpyAsync(output + rows * kCols, outSlot[slot], bytes, cudaMemcpyDeviceToHost, copyOut_))) {
				return false;
			}
		}
		if (!PTB_CUDA(cudaEventRecord(d2h_[slot], copyOut_))) { return false; }
		rows += static_cast<unsigned long long>(n);
		return true;
	};
	// one chunk slot: the previous chunk is completed (and its rows copied out of the shared workspace) before the
	// next is enqueued; two: chunk k - 1 is completed after chunk k is enqueued
	const bool serial = profiling_ || slots == 1;  // stage timing needs each chunk finished before the next starts
	bool ok = inputOnDevice || copyIn(0);
	for (uint64_t k = 0; ok && k < chunks; ++k) {
		const int ws = chunkSlot(k);  // workspace, compute stream, counters and events of this chunk
		const int b = framesOf(k);
		PlanWorkspace(Ws(ws), H, W, b, rowsCap, poolOf[ws]);
		const uint16_t* dImg = inputOnDevice ? input + first[k] * N : imgSlot(imgSlotOf(k));
		if (!inputOnDevice) { ok = PTB_CUDA(cudaStreamWaitEvent(St(ws), h2d_[imgSlotOf(k)], 0)); }
		// the rows of the chunk slot's previous chunk must be copied out before this chunk orders its rows there
		if (ok && !outputOnDevice && k >= static_cast<uint64_t>(slots)) { ok = PTB_CUDA(cudaStreamWaitEvent(St(ws), d2h_[ws], 0)); }
		outSlot[ws] = Ws(ws).sortedRows;
		double* dOut = outputOnDevice ? output : outSlot[ws];
		ok = ok && EnqueueChunk(ws, dImg, H, W, b, thr, ratio, maxPoints, fp, dOut, outputOnDevice, first[k], slots > 1 && k > 0);
		ok = ok && (inputOnDevice || PTB_CUDA(cudaEventRecord(imgFree_[imgSlotOf(k)], St(ws))));
		if (ok && !inputOnDevice && k + 1 < chunks) { ok = copyIn(k + 1); }
		if (ok && serial) { ok = complete(k); }
		else if (ok && k >= 1) { ok = complete(k - 1); }
	}
	if (ok && !serial && chunks > 0) { ok = complete(chunks - 1); }
	// work ordered after this call on the first compute stream also follows the second's
	if (ok && slots > 1) { ok = PTB_CUDA(cudaStreamWaitEvent(stream_, done_[1], 0)); }
	ok = ok && PTB_CUDA(cudaStreamSynchronize(copy_)) && PTB_CUDA(cudaStreamSynchronize(copyOut_));
	ok = ok && flushOut(static_cast<int>(outCopies & 1)) && flushOut(static_cast<int>((outCopies + 1) & 1));
	if (!ok) {
		cudaStreamSynchronize(stream_);
		cudaStreamSynchronize(stream1_);
		cudaStreamSynchronize(copy_);
		cudaStreamSynchronize(copyOut_);
		return -1;
	}
	for (uint32_t i = 0; i < truncated; ++i) {
		std::cerr << "[WARNING] Density is too high; some points are missed (output capacity exceeded).\n";
	}
	return static_cast<long long>(rows * kCols);
}

int EnvLanes()
{
	const char* env = std::getenv("PTB_MLE_LANES");
	return env ? std::atoi(env) : 0;
}

int EnvChunk()
{
	const char* env = std::getenv("PTB_MLE_CHUNK");
	return env ? std::max(1, std::atoi(env)) : 0;
}

// The ROI mapping of modes 6-8 for this chunk: PTB_MLE_LANES / PTB_MLE_CHUNK when set, else the autotuned choice of
// (mode, ROI, chunk size class); lanes stays 0 when that class has not been tuned yet.
void Engine::TunedMapping(FitParams& fp, int sizeClass) const
{
	const int envChunk = EnvChunk();
	if (const int env = EnvLanes()) {
		fp.lanes = env;
		fp.mle.chunk = envChunk ? envChunk : 1;
		return;
	}
	const int key = TuneKey(fp, sizeClass);
	for (const auto& t : tuned_) {
		if (t.key == key) {
			fp.lanes = t.lanes;
			fp.mle.chunk = envChunk ? envChunk : t.chunk;
			return;
		}
	}
	fp.lanes = 0;  // not tuned yet: the first chunk of this class with candidates tunes it
}

// Times the ROI mappings of modes 6-8 on this chunk's candidates - lanes per ROI (1: a thread per ROI through the
// four-launch pipeline; 2, 4, 8, 16: lane groups in the LM and polish; 32: a warp per ROI, one launch) and the work
// queue's chunk (candidates a lane takes at a time) - and keeps the fastest for (mode, ROI, chunk size class). Each
// choice runs once untimed before its timed run.
bool Engine::Autotune(FitParams& fp, const uint16_t* dImg, int H, int W, int slot, int sizeClass)
{
	Workspace& ws = Ws(slot);
	cudaStream_t st = St(slot);
	struct Choice {
		int lanes, chunk;
	};
	static const Choice kChoices[] = {{1, 1}, {1, 4}, {2, 1}, {4, 1}, {8, 1}, {16, 1}, {32, 1}};
	cudaEvent_t a, b;
	if (!PTB_CUDA(cudaEventCreate(&a)) || !PTB_CUDA(cudaEventCreate(&b))) { return false; }
	float best = 1e30f;
	Choice pick{32, 1};
	const int envChunk = EnvChunk();
	for (const Choice& c : kChoices) {
		if (envChunk && c.chunk != 1) { continue; }
		FitParams t = fp;
		t.lanes = c.lanes;
		t.mle.chunk = envChunk ? envChunk : c.chunk;
		t.mle.queue = ws.cnt->queue;
		// one untimed run first: the first launch of a kernel also loads its code, which is not what the choice costs
		if (!LaunchFit(dImg, H, W, ws.g.N, ws.cand, &ws.cnt->nfit, 0, ws.capRows, t, ws.rows, ws.fitFlag, precision_, st)) {
			return false;
		}
		cudaEventRecord(a, st);
		if (!LaunchFit(dImg, H, W, ws.g.N, ws.cand, &ws.cnt->nfit, 0, ws.capRows, t, ws.rows, ws.fitFlag, precision_, st)) {
			return false;
		}
		cudaEventRecord(b, st);
		if (!PTB_CUDA(cudaEventSynchronize(b))) { return false; }
		float ms = 0;
		cudaEventElapsedTime(&ms, a, b);
		if (ms < best) { best = ms; pick = c; }
	}
	cudaEventDestroy(a);
	cudaEventDestroy(b);
	fp.lanes = pick.lanes;
	fp.mle.chunk = envChunk ? envChunk : pick.chunk;
	tuned_.push_back({TuneKey(fp, sizeClass), pick.lanes, pick.chunk});
	return true;
}

int Engine::TunedMappings(int* out, int n, int skip) const
{
	int k = 0;
	for (int i = skip; i < static_cast<int>(tuned_.size()) && k < n; ++i, ++k) {
		const int key = tuned_[i].key;
		int* e = out + 5 * k;
		e[0] = key / (64 * 64);
		e[1] = (key / 64) % 64;
		e[2] = key % 64;
		e[3] = tuned_[i].lanes;
		e[4] = tuned_[i].chunk;
	}
	return k;
}

void Engine::GraphStats(uint64_t* out, int n)
{
	for (int k = 0; k < 3 && k < n; ++k) {
		if (out) { out[k] = graphCounts_[k]; }
		graphCounts_[k] = 0;
	}
}

void Engine::SegmentationStats(uint64_t* out, int n)
{
	for (int k = 0; k < 11 && k < n; ++k) {
		if (out) { out[k] = segCounts_[k]; }
		segCounts_[k] = 0;
	}
}

void Engine::StageTimes(double* ms, uint64_t* launches, int n)
{
	for (int k = 0; k < kStages && k < n; ++k) {
		if (ms) { ms[k] = stageMs_[k]; }
		if (launches) { launches[k] = stageLaunches_[k]; }
		stageMs_[k] = 0;
		stageLaunches_[k] = 0;
	}
}

void Engine::MleEvaluations(uint64_t* out, int n)
{
	for (int k = 0; k < 3 && k < n; ++k) {
		if (out) { out[k] = evalTotals_[k]; }
		evalTotals_[k] = 0;
	}
	if (n > 3) {
		// [3]: FP64 re-factorisations since the last call
		unsigned int fb = 0;
		if (fallbacks_ && Init() && PTB_CUDA(cudaStreamSynchronize(stream_)) &&
		    PTB_CUDA(cudaMemcpy(&fb, fallbacks_, sizeof(fb), cudaMemcpyDeviceToHost))) {
			cudaMemset(fallbacks_, 0, sizeof(unsigned int));
		}
		if (out) { out[3] = fb; }
	}
}

bool Engine::UploadSpline(FitParams& fp, const std::vector<double>& spline)
{
	if (fp.mode >= kMleGauss) {
		// [0] FP64 re-factorisation count, [1..2] work-queue counters of the persistent fit kernels
		if (!fallbacks_ && !PTB_CUDA(cudaMalloc(&fallbacks_, 4 * sizeof(unsigned int)))) { return false; }
		fp.mle.fallbacks = static_cast<unsigned int*>(fallbacks_);
		fp.mle.queue = static_cast<unsigned int*>(fallbacks_) + 1;
		fp.lanes = EnvLanes();  // 0: chosen per chunk by the autotuner
		fp.mle.chunk = EnvChunk() ? EnvChunk() : 1;
	}
	if (fp.mode != kMleSpline && fp.mode != kSplineEmccd) { return true; }
	// the same table as the last upload (a stack fitted chunk by chunk, or call after call): reuse the device copy
	const bool same = spline_ && splineCacheMode_ == fp.mode && splineCache_.size() == spline.size() &&
	                  std::memcmp(splineCache_.data(), spline.data(), spline.size() * sizeof(double)) == 0;
	if (!same) { splineCacheMode_ = -1; }  // the device copy is about to change: no longer the cached table
	if (fp.mode == kMleSpline) {
		// cell-major copies of the [64][cell] table: FP64 first, then FP32
		const size_t cells = static_cast<size_t>(fp.splineSize);
		if (same) {
			fp.mle.table64 = static_cast<const double*>(spline_);
			fp.mle.table = reinterpret_cast<const float*>(static_cast<const char*>(spline_) + cells * 64 * sizeof(double));
			return true;
		}
		std::vector<double> aos64(cells * 64);
		std::vector<float> aos32(cells * 64);
		for (size_t i = 0; i < 64; ++i) {
			for (size_t c = 0; c < cells; ++c) {
				aos64[c * 64 + i] = spline[i * cells + c];
				aos32[c * 64 + i] = static_cast<float>(spline[i * cells + c]);
			}
		}
		const size_t bytes64 = aos64.size() * sizeof(double), bytes32 = aos32.size() * sizeof(float);
		const size_t bytes = bytes64 + bytes32;
		if (bytes > splineBytes_) {
			if (spline_) { cudaFree(spline_); spline_ = nullptr; splineBytes_ = 0; }
			if (!PTB_CUDA(cudaMalloc(&spline_, bytes))) { return false; }
			splineBytes_ = bytes;
		}
		char* base = static_cast<char*>(spline_);
		if (!PTB_CUDA(cudaMemcpyAsync(base, aos64.data(), bytes64, cudaMemcpyHostToDevice, stream_))) { return false; }
		if (!PTB_CUDA(cudaMemcpyAsync(base + bytes64, aos32.data(), bytes32, cudaMemcpyHostToDevice, stream_))) { return false; }
		if (!PTB_CUDA(cudaStreamSynchronize(stream_))) { return false; }
		fp.mle.table64 = reinterpret_cast<const double*>(base);
		fp.mle.table = reinterpret_cast<const float*>(base + bytes64);
		splineCache_ = spline;
		splineCacheMode_ = fp.mode;
		return true;
	}
	// cell-major copy of the reference's [64][cell] table: one pixel's 64 coefficients become contiguous
	const size_t cells = static_cast<size_t>(fp.splineSize);
	if (same) {
		fp.coeffs = static_cast<const double*>(spline_);
		return true;
	}
	std::vector<double> aos(cells * 64);
	for (size_t i = 0; i < 64; ++i) {
		for (size_t c = 0; c < cells; ++c) { aos[c * 64 + i] = spline[i * cells + c]; }
	}
	const size_t bytes = aos.size() * sizeof(double);
	if (bytes > splineBytes_) {
		if (spline_) { cudaFree(spline_); spline_ = nullptr; splineBytes_ = 0; }
		if (!PTB_CUDA(cudaMalloc(&spline_, bytes))) { return false; }
		splineBytes_ = bytes;
	}
	if (!PTB_CUDA(cudaMemcpyAsync(spline_, aos.data(), bytes, cudaMemcpyHostToDevice, stream_))) { return false; }
	if (!PTB_CUDA(cudaStreamSynchronize(stream_))) { return false; }
	fp.coeffs = static_cast<const double*>(spline_);
	splineCache_ = spline;
	splineCacheMode_ = fp.mode;
	return true;
}

long long Engine::FitPositions(const uint16_t* input, const double* positions, uint64_t nPoints, double* output,
                               uint64_t height, uint64_t width, uint64_t planes, uint64_t fit, const double* fitParams)
{
	if (nPoints == 0) { return 0; }
	if (!Init()) { return -1; }
	FitParams fp;
	std::vector<double>& spline = splineIn_;
	if (!ParseFitParams(fit, fitParams, fp, spline)) { return -1; }
	if (!UploadSpline(fp, spline)) { return -1; }
	const size_t N = static_cast<size_t>(height) * width;
	std::vector<Cand> cands(nPoints);
	std::vector<double> localIdx(nPoints);
	std::vector<uint64_t> perPlane(planes, 0);
	std::vector<uint8_t> invalid(nPoints, 0);
	for (uint64_t i = 0; i < nPoints; ++i) {
		const double* pos = positions + i * 6;
		const double pl = pos[1];
		Cand c{};
		c.x = pos[2];
		c.y = pos[3];
		c.intensity = pos[4];
		c.surf = pos[5];
		if (!(pl >= 1.0) || static_cast<uint64_t>(pl) > planes) {
			// the reference indexes outside the stack here; this port returns a border-sentinel row instead
			invalid[i] = 1;
			c.x = -1.0;
			c.y = -1.0;
			c.frame = 0;
		}
		else {
			const uint64_t p = static_cast<uint64_t>(pl) - 1;
			c.frame = static_cast<int>(p);
			localIdx[i] = static_cast<double>(++perPlane[p]);
		}
		cands[i] = c;
	}
	const size_t imgBytes = N * planes * sizeof(uint16_t);
	if (!ReserveImage(imgBytes)) { return -1; }
	if (!PTB_CUDA(cudaMemcpyAsync(img_, input, imgBytes, cudaMemcpyHostToDevice, stream_))) { return -1; }
	Cand* dCand = nullptr;
	double* dRows = nullptr;
	uint8_t* dFlag = nullptr;
	bool ok = PTB_CUDA(cudaMallocAsync(&dCand, sizeof(Cand) * nPoints, stream_));
	ok = ok && PTB_CUDA(cudaMallocAsync(&dRows, sizeof(double) * kCols * nPoints, stream_));
	ok = ok && PTB_CUDA(cudaMallocAsync(&dFlag, nPoints, stream_));
	ok = ok && PTB_CUDA(cudaMemcpyAsync(dCand, cands.data(), sizeof(Cand) * nPoints, cudaMemcpyHostToDevice, stream_));
	// modes 6-8: a warp per ROI while the points fill the GPU a few times at most (shortest call), else a thread per ROI
	if (fp.mode >= kMleGauss && fp.lanes == 0) { fp.lanes = nPoints <= 148ull * 64 ? 32 : 1; }
	ok = ok && LaunchFit(static_cast<const uint16_t*>(img_), static_cast<int>(height), static_cast<int>(width),
	                     static_cast<long long>(N), dCand, nullptr, static_cast<uint32_t>(nPoints), static_cast<uint32_t>(nPoints),
	                     fp, dRows, dFlag, precision_, stream_);
	ok = ok && PTB_CUDA(cudaMemcpyAsync(output, dRows, sizeof(double) * kCols * nPoints, cudaMemcpyDeviceToHost, stream_));
	ok = ok && PTB_CUDA(cudaStreamSynchronize(stream_));
	if (dCand) { cudaFreeAsync(dCand, stream_); }
	if (dRows) { cudaFreeAsync(dRows, stream_); }
	if (dFlag) { cudaFreeAsync(dFlag, stream_); }
	if (!ok) { return -1; }
	for (uint64_t i = 0; i < nPoints; ++i) {
		double* r = output + i * kCols;
		if (invalid[i]) {
			r[cX] = positions[i * 6 + 2];
			r[cY] = positions[i * 6 + 3];
		}
		r[cId] = positions[i * 6 + 0];
		r[cPlane] = positions[i * 6 + 1];
		r[cIndex] = localIdx[i];
	}
	return static_cast<long long>(nPoints * kCols);
}

bool Engine::Planes(const uint16_t* input, double* output, uint64_t height, uint64_t width, uint64_t planes, int level)
{
	if (planes == 0 || height == 0 || width == 0) { return true; }
	if (!Init()) { return false; }
	const size_t N = static_cast<size_t>(height) * width;
	// chunk: input + output doubles within the budget
	const size_t perFrame = N * (sizeof(uint16_t) + sizeof(double));
	const uint64_t B = std::max<uint64_t>(1, std::min<uint64_t>(planes, budget_ / perFrame));
	if (!ReserveImage(N * B * sizeof(uint16_t))) { return false; }
	double* dOut = nullptr;
	if (!PTB_CUDA(cudaMallocAsync(&dOut, N * B * sizeof(double), stream_))) { return false; }
	bool ok = true;
	for (uint64_t z0 = 0; z0 < planes && ok; z0 += B) {
		const uint64_t b = std::min<uint64_t>(B, planes - z0);
		ok = ok && PTB_CUDA(cudaMemcpyAsync(img_, input + z0 * N, N * b * sizeof(uint16_t), cudaMemcpyHostToDevice, stream_));
		ok = ok && LaunchPlane(static_cast<const uint16_t*>(img_), dOut, static_cast<int>(height), static_cast<int>(width),
		                       static_cast<int>(b), level, stream_);
		ok = ok && PTB_CUDA(cudaMemcpyAsync(output + z0 * N, dOut, N * b * sizeof(double), cudaMemcpyDeviceToHost, stream_));
	}
	ok = ok && PTB_CUDA(cudaStreamSynchronize(stream_));
	cudaFreeAsync(dOut, stream_);
	cudaStreamSynchronize(stream_);
	return ok;
}

// AutoThreshold (lib/Palm.cpp:122-172): the standard deviations run on the host in the reference's summation order;
// each round's detection (fit 0, ratio 10) runs on the GPU.
double Engine::AutoThreshold(const uint16_t* input, uint64_t height, uint64_t width, const double* fitParams)
{
	if (!Init()) { return 0.0; }
	const size_t size = static_cast<size_t>(height) * width;
	if (size == 0 || fitParams == nullptr) { return 0.0; }
	const auto cap = static_cast<uint64_t>(0.2 * static_cast<double>(height * width) * kCols);
	const double halfRoi = fitParams[0] / 2;
	double mu = 0.0;
	for (size_t i = 0; i < size; ++i) { mu += input[i]; }
	mu /= static_cast<double>(size);
	double var = 0.0;
	for (size_t i = 0; i < size; ++i) { var += (input[i] - mu) * (input[i] - mu); }
	var /= static_cast<double>(size);
	double thr = std::sqrt(var);
	std::vector<double> rows(std::max<uint64_t>(cap, kCols));
	std::vector<char> mask(size);
	const size_t W = width, H = height;
	for (int iter = 0; iter < kThresholdIters; ++iter) {
		const long long n = Localize(input, false, rows.data(), false, cap, height, width, 1, thr, 10.0, 0, fitParams);
		if (n < 0) { return 0.0; }
		std::fill(mask.begin(), mask.end(), 0);
		for (long long k = 0; k < n / kCols; ++k) {
			const double px = rows[k * kCols + cX], py = rows[k * kCols + cY];
			const auto x0 = static_cast<size_t>(std::max(0, static_cast<int>(px - halfRoi)));
			const auto x1 = std::min(W, static_cast<size_t>(px + halfRoi));
			const auto y0 = static_cast<size_t>(std::max(0, static_cast<int>(py - halfRoi)));
			const auto y1 = std::min(H, static_cast<size_t>(py + halfRoi));
			for (size_t y = y0; y < y1; ++y) {
				for (size_t x = x0; x < x1; ++x) { mask[y * W + x] = 1; }
			}
		}
		size_t count = 0;
		double sum = 0;
		for (size_t j = 0; j < size; ++j) {
			if (!mask[j]) { sum += input[j]; ++count; }
		}
		if (count == 0) { break; }
		mu = sum / static_cast<double>(count);
		var = 0.0;
		for (size_t j = 0; j < size; ++j) {
			if (!mask[j]) { var += (input[j] - mu) * (input[j] - mu); }
		}
		var /= static_cast<double>(count);
		var = std::sqrt(var);
		if (std::abs(thr - var) <= 2.220446049250313e-16) { break; }
		thr = var;
	}
	return thr;
}

// Tracking over host buffers: [n][4] (Id, Plane, X, Y) -> [n][2] (Id, Track) in (Plane, Id) order.
bool Engine::Track(const double* input, uint64_t* output, uint64_t n, double maxDistance)
{
	if (n == 0) { return true; }
	if (!Init()) { return false; }
	double* dIn = nullptr;
	uint64_t* dOut = nullptr;
	bool ok = PTB_CUDA(cudaMallocAsync(&dIn, n * 4 * sizeof(double), stream_));
	ok = ok && PTB_CUDA(cudaMallocAsync(&dOut, n * 2 * sizeof(uint64_t), stream_));
	ok = ok && PTB_CUDA(cudaMemcpyAsync(dIn, input, n * 4 * sizeof(double), cudaMemcpyHostToDevice, stream_));
	ok = ok && TrackDevice(dIn, dOut, n, maxDistance, stream_);
	ok = ok && PTB_CUDA(cudaMemcpyAsync(output, dOut, n * 2 * sizeof(uint64_t), cudaMemcpyDeviceToHost, stream_));
	if (dIn) { cudaFreeAsync(dIn, stream_); }
	if (dOut) { cudaFreeAsync(dOut, stream_); }
	return PTB_CUDA(cudaStreamSynchronize(stream_)) && ok;
}

bool Engine::AstigEstimate(const double* input, double* output, uint64_t n, double pixelSize, const double* model, double zMax)
{
	if (n == 0) { return true; }
	if (!Init()) { return false; }
	const size_t bytes = static_cast<size_t>(n) * 2 * sizeof(double);
	double* dIn = nullptr;
	double* dOut = nullptr;
	bool ok = PTB_CUDA(cudaMallocAsync(&dIn, bytes, stream_));
	ok = ok && PTB_CUDA(cudaMallocAsync(&dOut, bytes, stream_));
	ok = ok && PTB_CUDA(cudaMemcpyAsync(dIn, input, bytes, cudaMemcpyHostToDevice, stream_));
	ok = ok && LaunchAstigEstimate(dIn, dOut, n, pixelSize, model, zMax, stream_);
	ok = ok && PTB_CUDA(cudaMemcpyAsync(output, dOut, bytes, cudaMemcpyDeviceToHost, stream_));
	if (dIn) { cudaFreeAsync(dIn, stream_); }
	if (dOut) { cudaFreeAsync(dOut, stream_); }
	return PTB_CUDA(cudaStreamSynchronize(stream_)) && ok;
}

// ---- engine pool --------------------------------------------------------------------------------------------
// Per device: the engines, which of them are leased, and the settings every engine of the device follows.
struct Pool {
	std::mutex mu;
	std::condition_variable freed;
	std::vector<std::unique_ptr<Engine>> engines;
	std::vector<char> busy;
	int leased = 0;
	int peak = 0;
	EngineSettings settings;
};

namespace {

constexpr int kMaxDevices = 64;

int MaxEngines()
{
	static const int n = [] {
		const char* e = std::getenv("PTB_MAX_ENGINES");
		const int v = e ? std::atoi(e) : 8;
		return std::max(1, std::min(v, 64));
	}();
	return n;
}

Pool& PoolFor(int dev)
{
	static Pool pools[kMaxDevices];
	return pools[std::max(0, std::min(dev, kMaxDevices - 1))];
}

int CurrentDevice()
{
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess) { dev = 0; }
	return dev;
}

}  // namespace

EngineSettings& SettingsFor() { return PoolFor(CurrentDevice()).settings; }

EngineLease::EngineLease()
{
	pool_ = &PoolFor(CurrentDevice());
	std::unique_lock<std::mutex> lock(pool_->mu);
	for (;;) {
		for (size_t i = 0; i < pool_->engines.size(); ++i) {
			if (!pool_->busy[i]) {
				index_ = static_cast<int>(i);
				break;
			}
		}
		if (index_ < 0 && static_cast<int>(pool_->engines.size()) < MaxEngines()) {
			pool_->engines.push_back(std::make_unique<Engine>());
			pool_->busy.push_back(0);
			index_ = static_cast<int>(pool_->engines.size()) - 1;
		}
		if (index_ >= 0) { break; }
		pool_->freed.wait(lock);
	}
	pool_->busy[index_] = 1;
	pool_->peak = std::max(pool_->peak, ++pool_->leased);
	engine_ = pool_->engines[index_].get();
	engine_->SetStrict(pool_->settings.strict.load());
	engine_->SetPrecision(pool_->settings.precision.load());
	engine_->SetProfiling(pool_->settings.profiling.load());
}

EngineLease::EngineLease(int index)
{
	pool_ = &PoolFor(CurrentDevice());
	std::unique_lock<std::mutex> lock(pool_->mu);
	if (index < 0 || index >= static_cast<int>(pool_->engines.size())) { return; }
	pool_->freed.wait(lock, [&] { return !pool_->busy[index]; });
	index_ = index;
	pool_->busy[index_] = 1;
	pool_->peak = std::max(pool_->peak, ++pool_->leased);
	engine_ = pool_->engines[index_].get();
}

EngineLease::~EngineLease()
{
	if (engine_ == nullptr) { return; }
	{
		std::lock_guard<std::mutex> lock(pool_->mu);
		pool_->busy[index_] = 0;
		--pool_->leased;
	}
	pool_->freed.notify_all();
}

void PoolStats(uint64_t* out, int n)
{
	Pool& p = PoolFor(CurrentDevice());
	std::lock_guard<std::mutex> lock(p.mu);
	const uint64_t v[2] = {p.engines.size(), static_cast<uint64_t>(p.peak)};
	for (int k = 0; k < 2 && k < n; ++k) {
		if (out) { out[k] = v[k]; }
	}
}

}  // namespace ptb
