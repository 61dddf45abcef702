// C ABI of the B200 localization engine (declared in include/palmtracer_b200.h). No exception crosses it: every
// entry point catches, records the message for PTB_LastError() and returns the reference's neutral value.
#include <cuda_runtime.h>

#include <algorithm>
#include <exception>
#include <iostream>

#include "../../include/palmtracer_b200.h"
#include "engine.h"
#include "tiff.h"

namespace {

void Report(const char* fn)
{
	std::cerr << "[PALMTracer-B200] " << fn << " failed: " << ptb::LastError() << "\n";
}

}  // namespace

extern "C" {

PTB_API uint64_t Localization(const uint16_t* input, double* output, uint64_t outputSize, uint64_t height, uint64_t width,
                              uint64_t planes, double thresholdVal, double watershedRatio, uint64_t fit, const double* fit_params)
{
	ptb::ClearError();
	try {
		ptb::EngineLease lease;
		ptb::Engine& e = *lease;
		const long long n = e.Localize(input, false, output, false, outputSize, height, width, planes, thresholdVal,
		                               watershedRatio, fit, fit_params);
		if (n < 0) { Report("Localization"); return 0; }
		return static_cast<uint64_t>(n);
	}
	catch (const std::exception& ex) {
		ptb::SetError(ex.what());
		Report("Localization");
		return 0;
	}
}

PTB_API uint64_t Fitting(const uint16_t* input, const double* positions, uint64_t nPoints, double* output, uint64_t /*outputSize*/,
                         uint64_t height, uint64_t width, uint64_t planes, uint64_t fit, const double* fit_params)
{
	ptb::ClearError();
	try {
		ptb::EngineLease lease;
		ptb::Engine& e = *lease;
		const long long n = e.FitPositions(input, positions, nPoints, output, height, width, planes, fit, fit_params);
		if (n < 0) { Report("Fitting"); return 0; }
		return static_cast<uint64_t>(n);
	}
	catch (const std::exception& ex) {
		ptb::SetError(ex.what());
		Report("Fitting");
		return 0;
	}
}

PTB_API void Wavelett(const uint16_t* input, double* output, uint64_t height, uint64_t width, uint64_t planes, uint64_t levelOutput)
{
	ptb::ClearError();
	try {
		if (planes == 0) { return; }
		if (levelOutput == 0) { levelOutput = 1; }
		const int level = static_cast<int>(std::min<uint64_t>(levelOutput - 1, 2));
		ptb::EngineLease lease;
		ptb::Engine& e = *lease;
		if (!e.Planes(input, output, height, width, planes, level)) { Report("Wavelett"); }
	}
	catch (const std::exception& ex) {
		ptb::SetError(ex.what());
		Report("Wavelett");
	}
}

PTB_API double AutoThreshold(const uint16_t* input, uint64_t height, uint64_t width, const double* fit_params)
{
	ptb::ClearError();
	try {
		ptb::EngineLease lease;
		ptb::Engine& e = *lease;
		const double t = e.AutoThreshold(input, height, width, fit_params);
		if (!ptb::LastError().empty()) { Report("AutoThreshold"); }
		return t;
	}
	catch (const std::exception& ex) {
		ptb::SetError(ex.what());
		Report("AutoThreshold");
		return 0.0;
	}
}

PTB_API void Astigmatism3DEstimation(const double* input, double* output, uint64_t size, double pixelSize, const double* model,
                                     double zMax)
{
	ptb::ClearError();
	try {
		if (size == 0) { return; }
		ptb::EngineLease lease;
		if (!lease->AstigEstimate(input, output, size, pixelSize, model, zMax)) { Report("Astigmatism3DEstimation"); }
	}
	catch (const std::exception& ex) {
		ptb::SetError(ex.what());
		Report("Astigmatism3DEstimation");
	}
}

PTB_API void Tracking(const double* input, uint64_t* output, uint64_t nPoints, double maxDistance)
{
	ptb::ClearError();
	try {
		ptb::EngineLease lease;
		if (!lease->Track(input, output, nPoints, maxDistance)) { Report("Tracking"); }
	}
	catch (const std::exception& ex) {
		ptb::SetError(ex.what());
		Report("Tracking");
	}
}

PTB_API uint64_t PTB_SplineCoefficients(const double* psf, uint64_t nx, uint64_t ny, uint64_t nz, const double* lambda, double* coeffs)
{
	ptb::ClearError();
	try {
		ptb::EngineLease lease;
		if (!lease->Init() || !ptb::SplineCoefficients(psf, nx, ny, nz, lambda, coeffs, lease->Stream())) {
			Report("PTB_SplineCoefficients");
			return 0;
		}
		return 64 * (nx - 1) * (ny - 1) * (nz - 1);
	}
	catch (const std::exception& ex) {
		ptb::SetError(ex.what());
		Report("PTB_SplineCoefficients");
		return 0;
	}
}

PTB_API uint64_t PTB_TrackingDevice(const double* d_input, uint64_t* d_output, uint64_t nPoints, double maxDistance, void* stream)
{
	ptb::ClearError();
	try {
		ptb::EngineLease lease;
		ptb::Engine& e = *lease;
		if (!e.Init()) { Report("PTB_TrackingDevice"); return 0; }
		if (!ptb::TrackDevice(d_input, d_output, nPoints, maxDistance, static_cast<cudaStream_t>(stream))) {
			Report("PTB_TrackingDevice");
			return 0;
		}
		return 2 * nPoints;
	}
	catch (const std::exception& ex) {
		ptb::SetError(ex.what());
		Report("PTB_TrackingDevice");
		return 0;
	}
}

PTB_API int PTB_TiffInfo(const char* path, uint64_t* width, uint64_t* height, uint64_t* planes)
{
	ptb::ClearError();
	try {
		ptb::TiffStack t;
		if (!t.Open(path)) { Report("PTB_TiffInfo"); return 0; }
		if (width) { *width = t.Width(); }
		if (height) { *height = t.Height(); }
		if (planes) { *planes = t.Planes(); }
		return 1;
	}
	catch (const std::exception& ex) {
		ptb::SetError(ex.what());
		Report("PTB_TiffInfo");
		return 0;
	}
}

PTB_API uint64_t PTB_TiffRead(const char* path, uint16_t* output, uint64_t first, uint64_t count)
{
	ptb::ClearError();
	try {
		ptb::TiffStack t;
		if (!t.Open(path) || !t.Read(first, count, output)) { Report("PTB_TiffRead"); return 0; }
		return count;
	}
	catch (const std::exception& ex) {
		ptb::SetError(ex.what());
		Report("PTB_TiffRead");
		return 0;
	}
}

PTB_API uint64_t PTB_LocalizationTiff(const char* path, double* output, uint64_t outputSize, double thresholdVal,
                                      double watershedRatio, uint64_t fit, const double* fit_params)
{
	ptb::ClearError();
	try {
		ptb::TiffStack t;
		if (!t.Open(path)) { Report("PTB_LocalizationTiff"); return 0; }
		const ptb::Engine::PageSource source = [&t](uint64_t first, uint64_t count, uint16_t* dst) { return t.Read(first, count, dst); };
		ptb::EngineLease lease;
		ptb::Engine& e = *lease;
		const long long n = e.Localize(nullptr, false, output, false, outputSize, t.Height(), t.Width(), t.Planes(), thresholdVal,
		                               watershedRatio, fit, fit_params, &source);
		if (n < 0) { Report("PTB_LocalizationTiff"); return 0; }
		return static_cast<uint64_t>(n);
	}
	catch (const std::exception& ex) {
		ptb::SetError(ex.what());
		Report("PTB_LocalizationTiff");
		return 0;
	}
}

PTB_API uint64_t PTB_LocalizationDevice(const uint16_t* d_input, double* d_output, uint64_t outputSize, uint64_t height,
                                        uint64_t width, uint64_t planes, double thresholdVal, double watershedRatio, uint64_t fit,
                                        const double* fit_params, void* stream)
{
	ptb::ClearError();
	try {
		ptb::EngineLease lease;
		ptb::Engine& e = *lease;
		if (!e.Init()) { Report("PTB_LocalizationDevice"); return 0; }
		const cudaStream_t own = e.Stream();
		cudaStream_t user = static_cast<cudaStream_t>(stream);
		// order the engine's stream after the caller's work, and the caller's stream after the engine's
		cudaEvent_t ev;
		if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) { return 0; }
		cudaEventRecord(ev, user);
		cudaStreamWaitEvent(own, ev, 0);
		const long long n = e.Localize(d_input, true, d_output, true, outputSize, height, width, planes, thresholdVal,
		                               watershedRatio, fit, fit_params);
		cudaEventRecord(ev, own);
		cudaStreamWaitEvent(user, ev, 0);
		cudaEventDestroy(ev);
		if (n < 0) { Report("PTB_LocalizationDevice"); return 0; }
		return static_cast<uint64_t>(n);
	}
	catch (const std::exception& ex) {
		ptb::SetError(ex.what());
		Report("PTB_LocalizationDevice");
		return 0;
	}
}

PTB_API uint64_t PTB_FittingDeviceNoAlloc(const uint16_t* d_input, const double* d_positions, uint64_t nPoints,
                                          double* d_output, uint64_t height, uint64_t width, uint64_t planes, uint64_t fit,
                                          const double* fit_params, void* stream)
{
	ptb::ClearError();
	try {
		const int precision = ptb::SettingsFor().precision.load();  // a setting; initialises no device state
		const long long n = ptb::FittingDeviceNoAlloc(d_input, d_positions, nPoints, d_output, height, width, planes, fit,
		                                              fit_params, precision, ptb::EnvLanes(), static_cast<cudaStream_t>(stream));
		if (n < 0) { Report("PTB_FittingDeviceNoAlloc"); return 0; }
		return static_cast<uint64_t>(n);
	}
	catch (const std::exception& ex) {
		ptb::SetError(ex.what());
		Report("PTB_FittingDeviceNoAlloc");
		return 0;
	}
}

PTB_API int PTB_SetSegmentationMode(int mode)
{
	return ptb::SettingsFor().strict.exchange(mode == 1 || mode == 2 ? mode : 0);
}

PTB_API int PTB_SetFitPrecision(int mode) { return ptb::SettingsFor().precision.exchange(mode < 0 ? 0 : (mode > 2 ? 2 : mode)); }

PTB_API const char* PTB_LastError(void) { return ptb::LastError().c_str(); }

PTB_API uint64_t PTB_KernelLaunchCount(void) { return ptb::LaunchCount(); }

PTB_API double PTB_MeasureFmaPeak(int fp64)
{
	ptb::ClearError();
	return ptb::MeasureFmaPeak(fp64);
}

PTB_API int PTB_SetProfiling(int enable) { return ptb::SettingsFor().profiling.exchange(enable ? 1 : 0); }

PTB_API void PTB_StageTimes(double* ms, uint64_t* launches, int n)
{
	constexpr int kMax = 16;
	double sumMs[kMax] = {};
	uint64_t sumL[kMax] = {};
	n = std::max(0, std::min(n, kMax));
	for (int i = 0;; ++i) {
		ptb::EngineLease lease(i);
		if (!lease) { break; }
		double m[kMax] = {};
		uint64_t l[kMax] = {};
		lease->StageTimes(m, l, n);
		for (int k = 0; k < n; ++k) { sumMs[k] += m[k]; sumL[k] += l[k]; }
	}
	for (int k = 0; k < n; ++k) {
		if (ms) { ms[k] = sumMs[k]; }
		if (launches) { launches[k] = sumL[k]; }
	}
}

PTB_API int PTB_ServerStart(int slots, uint64_t budgetBytes)
{
	ptb::ClearError();
	try {
		if (ptb::ServerStart(slots, budgetBytes)) { return 1; }
	}
	catch (const std::exception& ex) {
		ptb::SetError(ex.what());
	}
	Report("PTB_ServerStart");
	return 0;
}

PTB_API void PTB_ServerStop(void)
{
	try {
		ptb::ServerStop();
	}
	catch (const std::exception& ex) {
		ptb::SetError(ex.what());
		Report("PTB_ServerStop");
	}
}

PTB_API uint64_t PTB_SubmitStack(const uint16_t* input, double* output, uint64_t outputSize, uint64_t height, uint64_t width,
                                 uint64_t planes, double thresholdVal, double watershedRatio, uint64_t fit, const double* fit_params)
{
	ptb::ClearError();
	try {
		const uint64_t id = ptb::SubmitStack(input, output, outputSize, height, width, planes, thresholdVal, watershedRatio, fit,
		                                     fit_params, ptb::FitParamCount(fit, fit_params));
		if (id == 0) { Report("PTB_SubmitStack"); }
		return id;
	}
	catch (const std::exception& ex) {
		ptb::SetError(ex.what());
		Report("PTB_SubmitStack");
		return 0;
	}
}

PTB_API void PTB_ServerFuseStats(uint64_t* counts, int n) { ptb::ServerFuseStats(counts, n); }

PTB_API int PTB_PollStack(uint64_t ticket)
{
	try {
		return ptb::PollStack(ticket);
	}
	catch (const std::exception&) {
		return -1;
	}
}

PTB_API int64_t PTB_StackResult(uint64_t ticket, double* times)
{
	ptb::ClearError();
	try {
		const long long n = ptb::StackResult(ticket, times);
		if (n < 0) { Report("PTB_StackResult"); }
		return n;
	}
	catch (const std::exception& ex) {
		ptb::SetError(ex.what());
		Report("PTB_StackResult");
		return -1;
	}
}

}  // extern "C"

namespace {

// Sums a counter diagnostic over every engine of the current device's pool (each read resets that engine's counters).
template <typename Fn>
void SumOverEngines(uint64_t* counts, int n, Fn read)
{
	constexpr int kMax = 16;
	uint64_t sum[kMax] = {};
	n = std::max(0, std::min(n, kMax));
	for (int i = 0;; ++i) {
		ptb::EngineLease lease(i);
		if (!lease) { break; }
		uint64_t v[kMax] = {};
		read(*lease, v, n);
		for (int k = 0; k < n; ++k) { sum[k] += v[k]; }
	}
	for (int k = 0; k < n && counts; ++k) { counts[k] = sum[k]; }
}

}  // namespace

extern "C" {

PTB_API void PTB_MleEvaluations(uint64_t* counts, int n)
{
	SumOverEngines(counts, n, [](ptb::Engine& e, uint64_t* v, int k) { e.MleEvaluations(v, k); });
}

PTB_API void PTB_DetectStagingStats(uint64_t* counts, int n)
{
	ptb::DetectStagingStats(counts, n);
}

PTB_API void PTB_GraphStats(uint64_t* counts, int n)
{
	SumOverEngines(counts, n, [](ptb::Engine& e, uint64_t* v, int k) { e.GraphStats(v, k); });
}

PTB_API void PTB_SegmentationStats(uint64_t* counts, int n)
{
	SumOverEngines(counts, n, [](ptb::Engine& e, uint64_t* v, int k) { e.SegmentationStats(v, k); });
}

PTB_API void PTB_EnginePoolStats(uint64_t* counts, int n) { ptb::PoolStats(counts, n); }

PTB_API int PTB_MleMappings(int* entries, int n)
{
	int written = 0;
	for (int i = 0; written < n; ++i) {
		ptb::EngineLease lease(i);
		if (!lease) { break; }
		written += lease->TunedMappings(entries + 5 * written, n - written, 0);
	}
	return written;
}

}  // extern "C"
