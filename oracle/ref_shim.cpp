// Test infrastructure only: C entry points over the UNMODIFIED reference CPU library.
//
// This file is compiled together with the reference's own sources (lib/Palm.cpp, lib/localization/*.cpp,
// lib/fit/*.cpp, lib/signal_processing/Matrix.cpp) into oracle/_ref/libptref.so by oracle/build_ref.sh.
// It is the checker and the timed CPU baseline; nothing in the product links or calls it.
//
// The four wrappers mirror the reference exports one for one:
//   ref_Localization  -> CPU/main.cpp:112-121 (Localization)
//   ref_Fitting       -> CPU/main.cpp:141-148 (Fitting)
//   ref_Wavelett      -> CPU/main.cpp:257-284 (Wavelett)
//   ref_AutoThreshold -> CPU/main.cpp:75-85   (AutoThreshold)
// ref_Astig3DEstimation mirrors CPU/main.cpp:324-353, ref_Tracking CPU/main.cpp:159-164 (Tracking). The remaining entry points expose intermediate
// products (wavelet planes, segmentation candidates, label map) for bitwise checks of each stage.
#include <omp.h>

#include <algorithm>
#include <array>
#include <cstdint>
#include <cstring>
#include <vector>

#include "Palm.hpp"
#include "fit/AstigFit.hpp"
#include "localization/ATrous.hpp"
#include "localization/Segmentation2D.hpp"
#include "tracking/Tracks.hpp"

namespace pt = palm_tracer;

extern "C" {

void ref_SetThreads(int n)
{
	omp_set_dynamic(1);
	if (n > 0) { omp_set_num_threads(n); }
}

int ref_MaxThreads(void) { return omp_get_max_threads(); }

uint64_t ref_Localization(const uint16_t* input, double* output, uint64_t outputSize, uint64_t height, uint64_t width,
                          uint64_t planes, double thresholdVal, double watershedRatio, uint64_t fit, const double* fitParams)
{
	const pt::Vec3I dim{.x = width, .y = height, .z = planes};
	const pt::Palm palm(input, output, outputSize, dim, thresholdVal, watershedRatio, fit, fitParams);
	return static_cast<uint64_t>(palm.Processing());
}

uint64_t ref_Fitting(const uint16_t* input, const double* positions, uint64_t nPoints, double* output, uint64_t outputSize,
                     uint64_t height, uint64_t width, uint64_t planes, uint64_t fit, const double* fitParams)
{
	const pt::Vec3I dim{.x = width, .y = height, .z = planes};
	return pt::Palm::FitLocalizations(input, positions, nPoints, output, outputSize, dim, fit, fitParams);
}

void ref_Wavelett(const uint16_t* input, double* output, uint64_t height, uint64_t width, uint64_t planes, uint64_t level)
{
	if (planes == 0) { return; }
	if (level == 0) { level = 1; }
	const pt::Vec2I dim{.x = width, .y = height};
	const uint64_t size = dim.GetSize();
	const uint64_t lvl  = std::min<uint64_t>(level - 1, pt::N_PLANES - 1);
	pt::localization::ATrous decomposition(dim);
	for (uint64_t i = 0; i < planes; ++i) {
		decomposition.Process(input + i * size);
		std::copy_n(decomposition.wDecomp_[lvl].data(), size, output + i * size);
	}
}

double ref_AutoThreshold(const uint16_t* input, uint64_t height, uint64_t width, const double* fitParams)
{
	const auto cap = static_cast<uint64_t>(0.2 * static_cast<double>(height * width) * pt::localization_columns::Count);
	std::vector<double> points(cap);
	const pt::Vec3I dim{.x = width, .y = height, .z = 1};
	auto palm = pt::Palm(input, points.data(), cap, dim, 0, 10, 0, fitParams);
	return palm.AutoThreshold();
}

// All N_PLANES planes of one frame: planes[k * H * W + p].
void ref_Planes(const uint16_t* frame, uint64_t height, uint64_t width, double* planes)
{
	const pt::Vec2I dim{.x = width, .y = height};
	const pt::localization::ATrous decomposition(frame, dim);
	for (size_t k = 0; k < pt::N_PLANES; ++k) {
		std::copy_n(decomposition.wDecomp_[k].data(), dim.GetSize(), planes + k * dim.GetSize());
	}
}

// Segmentation candidates of one frame, in label order: rows of (x_, y_, intensity_, surf_).
// Returns the number of candidates; writes at most `capacity` rows.
uint64_t ref_Candidates(const uint16_t* frame, uint64_t height, uint64_t width, double threshold, double ratio,
                        double* rows, uint64_t capacity)
{
	const pt::Vec2I dim{.x = width, .y = height};
	const pt::localization::ATrous decomposition(frame, dim);
	const pt::localization::Segmentation2D seg(decomposition, threshold, ratio);
	const auto& infos = seg.Infos();
	for (size_t i = 0; i < infos.size() && i < capacity; ++i) {
		rows[4 * i + 0] = infos[i].x_;
		rows[4 * i + 1] = infos[i].y_;
		rows[4 * i + 2] = infos[i].intensity_;
		rows[4 * i + 3] = infos[i].surf_;
	}
	return infos.size();
}

// Same as ref_Candidates, but segmenting a caller-given potential (replaces wavelet plane 1), as the
// reference segmentation tests do (Tests_CPU/test_loc_Segmentation2D.cpp:13-19).
uint64_t ref_CandidatesFromPotential(const double* potential, uint64_t height, uint64_t width, double threshold, double ratio,
                                     double* rows, uint64_t capacity)
{
	const pt::Vec2I dim{.x = width, .y = height};
	std::vector<uint16_t> black(dim.GetSize(), 0);
	pt::localization::ATrous decomposition(black.data(), dim);
	std::copy_n(potential, dim.GetSize(), decomposition.wDecomp_[pt::PLANE_ID].begin());
	const pt::localization::Segmentation2D seg(decomposition, threshold, ratio);
	const auto& infos = seg.Infos();
	for (size_t i = 0; i < infos.size() && i < capacity; ++i) {
		rows[4 * i + 0] = infos[i].x_;
		rows[4 * i + 1] = infos[i].y_;
		rows[4 * i + 2] = infos[i].intensity_;
		rows[4 * i + 3] = infos[i].surf_;
	}
	return infos.size();
}

void ref_Astig3DEstimation(const double* input, double* output, uint64_t size, double pixelSize, const double* model, double zMax)
{
	std::vector<pt::Vec2D> sig(size);
	for (uint64_t i = 0; i < size; ++i) { sig[i] = {.x = input[2 * i], .y = input[2 * i + 1]}; }
	const pt::fit::astig_model m = {std::array{model[0], model[1], model[2], model[3], model[4]},
	                                std::array{model[5], model[6], model[7], model[8], model[9]}};
	const pt::fit::AstigFit fit(pixelSize);
	const auto res = fit.Estimate(m, sig, std::array{-zMax, zMax});
	for (uint64_t i = 0; i < size; ++i) {
		output[2 * i]     = res[i].x;
		output[2 * i + 1] = res[i].y;
	}
}

uint64_t ref_Tracking(const double* input, uint64_t* output, uint64_t nPoints, double maxDistance)
{
	return pt::tracking::Tracks::Tracking(input, output, nPoints, maxDistance);
}
}
