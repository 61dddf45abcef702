// Host engine of the B200 localization path. Each device has a pool of engines: a call leases one for its duration
// (EngineLease), so concurrent callers run on their own streams and workspaces.
#pragma once

#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "pt_common.cuh"

namespace ptb {

bool ParseFitParams(uint64_t fit, const double* fp, FitParams& out, std::vector<double>& splineHost);
long long FittingDeviceNoAlloc(const uint16_t* dStack, const double* dPositions, uint64_t nPoints, double* dOutput,
                               uint64_t height, uint64_t width, uint64_t planes, uint64_t fit, const double* fitParams,
                               int precision, int lanes, cudaStream_t st);
int EnvLanes();
int EnvChunk();
// Serving (server.cpp)
bool ServerStart(int slots, uint64_t budgetBytes);
void ServerStop();
uint64_t SubmitStack(const uint16_t* input, double* output, uint64_t outputSize, uint64_t height, uint64_t width, uint64_t planes,
                     double thr, double ratio, uint64_t fit, const double* fitParams, size_t nParams);
int PollStack(uint64_t id);
// [fused fit launches, chunks fitted by them] of the running server (zeros without one).
void ServerFuseStats(uint64_t* out, int n);
long long StackResult(uint64_t id, double* times);
// Number of fit_params entries the given fit mode reads (0 for mode 0 or an unknown mode).
size_t FitParamCount(uint64_t fit, const double* fp);
uint64_t LaunchCount();
bool TrackDevice(const double* dIn, uint64_t* dOut, uint64_t nPoints, double maxDistance, cudaStream_t st);
double MeasureFmaPeak(int fp64);
bool SplineCoefficients(const double* volume, uint64_t nx, uint64_t ny, uint64_t nz, const double* lambda, double* out, cudaStream_t st);

// A chunk's maximum-likelihood fit handed to a stage outside the engine (the serving layer's fused fits). The
// candidates and the frames are ready on `stream`; the stage must fill rows[0, *count) and order that work before
// whatever `stream` runs next before it returns.
struct FitJob {
	cudaStream_t stream;
	FitImage image;
	const Cand* cands;
	const uint32_t* count;  // device
	uint32_t cap;
	double* rows;           // [cap][18]
	FitParams fp;
};
using FitHook = std::function<bool(const FitJob&)>;

class Engine {
public:
	Engine();
	~Engine();
	Engine(const Engine&) = delete;
	Engine& operator=(const Engine&) = delete;

	// Fills frames [first, first + count) of the stack into a host buffer ([count][height][width]); false on error.
	using PageSource = std::function<bool(uint64_t first, uint64_t count, uint16_t* dst)>;
	// Localization over host or device buffers; returns doubles written or -1 (error recorded). With a page source
	// (input null, host output), each chunk's frames are produced into pinned staging on the host while the previous
	// chunk computes.
	long long Localize(const uint16_t* input, bool inputOnDevice, double* output, bool outputOnDevice, uint64_t outputSize,
	                   uint64_t height, uint64_t width, uint64_t planes, double thr, double ratio, uint64_t fit,
	                   const double* fitParams, const PageSource* source = nullptr);
	long long FitPositions(const uint16_t* input, const double* positions, uint64_t nPoints, double* output, uint64_t height,
	                       uint64_t width, uint64_t planes, uint64_t fit, const double* fitParams);
	bool Planes(const uint16_t* input, double* output, uint64_t height, uint64_t width, uint64_t planes, int level);
	double AutoThreshold(const uint16_t* input, uint64_t height, uint64_t width, const double* fitParams);
	// Astigmatism3DEstimation over host buffers: [n][2] widths (px) -> [n][2] (z nm, score).
	bool AstigEstimate(const double* input, double* output, uint64_t n, double pixelSize, const double* model, double zMax);
	// Tracking over host buffers: [n][4] (Id, Plane, X, Y) -> [n][2] (Id, Track) in (Plane, Id) order.
	bool Track(const double* input, uint64_t* output, uint64_t n, double maxDistance);

	int SetStrict(int s) { const int o = strict_; strict_ = s; return o; }
	int SetProfiling(int p) { const int o = profiling_; profiling_ = p; return o; }
	void StageTimes(double* ms, uint64_t* launches, int n);
	void MleEvaluations(uint64_t* out, int n);
	// [chunks captured into graphs, chunks replayed from graphs, chunks launched directly] since the last call.
	void GraphStats(uint64_t* out, int n);
	// [frames segmented, frames flooded again frame-wide after failing the exactness test] since the last call.
	void SegmentationStats(uint64_t* out, int n);
	// The autotuned ROI mappings of modes 6-8: up to n entries of (mode, roi, chunk size class, lanes, chunk) after
	// the first `skip` entries; returns the entries written.
	int TunedMappings(int* out, int n, int skip) const;
	int SetPrecision(int p) { const int o = precision_; precision_ = p; return o; }
	int Precision() const { return precision_; }
	cudaStream_t Stream() const { return stream_; }
	// Device-memory budget of the chunk workspace (bytes); 0 = a quarter of free memory at first use, at most 48 GiB
	// (or PTB_WORKSPACE_MB). Takes effect at the engine's first call.
	void SetBudget(size_t bytes) { fixedBudget_ = bytes; }
	size_t Budget() const { return budget_; }
	// Device bytes a Localize call of this shape would hold (chunk workspace and staging), for admission control.
	size_t EstimateBytes(uint64_t height, uint64_t width, uint64_t planes, uint64_t outputSize) const;
	void SetStream(cudaStream_t s) { stream_ = s; }
	// Modes 6-8 fit through `hook` instead of the engine's own launches (empty: the engine fits).
	void SetFitHook(FitHook hook) { fitHook_ = std::move(hook); }
	bool Init();

private:
	bool Reserve(int H, int W, int B, uint32_t rowsCap, int slots);
	bool ReserveImage(size_t bytes);
	bool UploadSpline(FitParams& fp, const std::vector<double>& spline);
	void TunedMapping(FitParams& fp, int sizeClass) const;
	bool Autotune(FitParams& fp, const uint16_t* dImg, int H, int W, int slot, int sizeClass);
	int ChunkFrames(int H, int W, uint64_t planes, uint32_t maxPoints, size_t budget) const;
	// Chunk size and number of concurrent chunk slots (2 when the stack needs more than one chunk).
	void ChunkPlan(int H, int W, uint64_t planes, uint32_t maxPoints, int& B, int& slots) const;
	Workspace& Ws(int slot) { return slot ? ws1_ : ws_; }
	cudaStream_t St(int slot) const { return slot ? stream1_ : stream_; }
	// One chunk of B frames on the compute stream: detection, segmentation, fits, ordering into dOut (at dOut +
	// rows so far when offsetOut), counters copied to the slot's pinned buffer, completion event recorded.
	// afterOther: the chunk orders its rows after the chunk in flight on the other slot (its Ids continue from it).
	bool EnqueueChunk(int slot, const uint16_t* dImg, int H, int W, int B, double thr, double ratio, uint32_t maxPoints,
	                  const FitParams& fp, double* dOut, bool offsetOut, unsigned long long planeBase, bool afterOther);
	// Executable graphs of chunk launch chains, per chunk slot, keyed by every argument the chain's launches take.
	struct GraphEntry {
		std::vector<uint64_t> key;
		cudaGraphExec_t exec;
		uint64_t launches;  // kernels in the graph
		uint64_t lastUse;
		bool fresh;         // captured, not replayed yet (its launches were counted while recording)
	};
	static constexpr size_t kGraphsPerSlot = 32;
	GraphEntry* FindGraph(int slot, const std::vector<uint64_t>& key);
	GraphEntry* CaptureGraph(int slot, std::vector<uint64_t> key, const std::function<bool()>& launch);
	// Waits for the slot's chunk; returns its row count or -1 (error recorded).
	long long CompleteChunk(int slot, uint32_t* truncatedFrames);

	int device_ = 0;
	cudaStream_t stream_ = nullptr;
	cudaStream_t copy_ = nullptr;            // host-to-device copies that overlap the compute streams
	cudaStream_t copyOut_ = nullptr;         // device-to-host copies (the other direction of the link, concurrently)
	cudaStream_t stream1_ = nullptr;         // second compute stream (second chunk slot)
	cudaEvent_t sortDone_[2] = {};           // per chunk slot: its rows are ordered (Ids of the next chunk follow)
	cudaEvent_t fork_ = nullptr;              // start of a two-slot call on the first compute stream
	std::vector<GraphEntry> graphs_[2];
	std::vector<std::vector<uint64_t>> seen_[2];  // chains launched once directly (the next occurrence is captured)
	uint64_t graphClock_ = 0;
	uint64_t graphCounts_[3] = {};            // captured, replayed, direct
	uint64_t segCounts_[11] = {};             // frames segmented, flooded frame-wide, given the rank test, re-flooded;
	                                          // flooded frame-wide by reason (RouteReason)
	bool useGraphs_ = true;                   // PTB_GRAPHS=0 launches every chunk directly
	bool graphsOff_ = false;                  // a capture failed: direct launches from then on
	Workspace ws1_{};                        // second chunk slot's workspace and pool
	void* pool1_ = nullptr;
	size_t pool1Bytes_ = 0;
	cudaEvent_t h2d_[3] = {}, imgFree_[3] = {};  // per frame staging slot on the device: copied in, read by its chunk
	cudaEvent_t done_[2] = {}, d2h_[2] = {};     // per chunk slot: chunk finished, its rows copied out
	Counters* hostCnt_ = nullptr;             // pinned, one per chunk slot
	unsigned long long* rowBase_ = nullptr;   // device: rows written by the earlier chunks of the current call
	size_t budget_ = 0;
	size_t fixedBudget_ = 0;
	void* pool_ = nullptr;
	size_t poolBytes_ = 0;
	void* img_ = nullptr;
	size_t imgBytes_ = 0;
	void* hostStage_ = nullptr;               // pinned frame staging of page sources (two slots)
	size_t hostStageBytes_ = 0;
	void* hostOut_[2] = {};                   // pinned row staging for pageable output (two buffers)
	size_t hostOutBytes_[2] = {};
	cudaEvent_t outEv_[2] = {};               // a staged row copy reached hostOut_
	void* spline_ = nullptr;
	std::vector<double> splineIn_;            // the call's spline table as given (reused between calls)
	std::vector<double> splineCache_;         // the table behind spline_ (its upload is skipped when unchanged)
	int splineCacheMode_ = -1;
	void* fallbacks_ = nullptr;
	struct Tuned {
		int key;    // (mode * 64 + roi) * 64 + chunk size class
		int lanes;  // lanes per ROI
		int chunk;  // work-queue chunk
	};
	std::vector<Tuned> tuned_;
	size_t splineBytes_ = 0;
	Workspace ws_{};
	FitHook fitHook_;
	int strict_ = 0;
	int precision_ = 0;
	int profiling_ = 0;
	// profiling: detect, segment, fit, finish, copies, then the phases of a modes 6-8 fit (initial values, LM, polish,
	// FP64 likelihood and CRLB)
	static constexpr int kStages = 9;
	cudaEvent_t ev_[6] = {};
	cudaEvent_t mleEv_[5] = {};
	double stageMs_[kStages] = {};
	uint64_t stageLaunches_[kStages] = {};
	unsigned long long* evalDev_ = nullptr;      // device counters of model evaluations (profiling)
	unsigned long long evalTotals_[3] = {};      // FP32 LM, FP32 polish, FP64
	// profiling bookkeeping of the chunk in flight
	uint64_t pendLaunches_[kStages] = {};
	bool pendMleProf_ = false;
	int pendLanes_ = 0;
};

// Settings that PTB_SetSegmentationMode / PTB_SetFitPrecision / PTB_SetProfiling change for every engine of a device
// (applied to an engine each time it is leased).
struct EngineSettings {
	std::atomic<int> strict{0};
	std::atomic<int> precision{0};
	std::atomic<int> profiling{0};
};
EngineSettings& SettingsFor();  // the current device's

// One engine of the current device's pool, held for one call. A lease takes the first idle engine, creates a new one
// when every engine is busy and the pool holds fewer than PTB_MAX_ENGINES (default 8), and otherwise waits for one to
// be released; so concurrent callers get their own engines (own CUDA streams, chunk workspaces, graphs and autotuned
// choices) and overlap on the device, and sequential callers keep reusing the first engine. Lease(index) takes that
// specific engine (waiting while it is busy), for diagnostics that visit every engine; it is empty when the pool has
// no such engine.
class EngineLease {
public:
	EngineLease();
	explicit EngineLease(int index);
	~EngineLease();
	EngineLease(const EngineLease&) = delete;
	EngineLease& operator=(const EngineLease&) = delete;
	Engine& operator*() const { return *engine_; }
	Engine* operator->() const { return engine_; }
	explicit operator bool() const { return engine_ != nullptr; }

private:
	struct Pool* pool_ = nullptr;
	int index_ = -1;
	Engine* engine_ = nullptr;
};

// [engines in the current device's pool, most engines leased at the same time] (diagnostics).
void PoolStats(uint64_t* out, int n);

// [detection launches staged by the TMA, by per-thread loads] since the last call, whole process (diagnostics).
void DetectStagingStats(uint64_t* out, int n);

}  // namespace ptb
