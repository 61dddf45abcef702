/*
 * PALMTracer localization hot path on one NVIDIA B200 (sm_100a): public C ABI.
 *
 * The first four entry points are drop-in replacements for the exports of the PALMTracer CPU library
 * (tmonseigne/PALMTracer-cpp 1.3.0, CPU/PALMTracer.def:3-13, declared with PT_API in lib/ExportAPI.hpp:21-30):
 * same names, argument meaning, buffer layouts, return values and error behaviour (no exception ever crosses the
 * ABI; bad input yields 0 / no output, failed fits yield the usual -1 sentinel rows). All buffers are caller-owned
 * HOST memory; the library keeps no pointer after a call returns.
 *
 * Layouts (lib/Constants.hpp:31-64):
 *   input       uint16 [planes][height][width], x fastest
 *   output      float64 rows of 18 columns: Id, Plane, Index, Channel, X, Y, Z, Integrated intensity, SigmaX, SigmaY,
 *               Theta, QualityXY, QualityZ, Amplitude, Offset, SegIntensity, Surface, Circularity
 *   positions   float64 rows of 6 columns: Id, Plane (1-based), X, Y, SegIntensity, Surface
 *   fit_params  Gaussian modes 1-4: [roi, sigmaX, sigmaY, theta]
 *               spline mode 5:      [roi, sx, sy, sz, deltaZ, 64*sx*sy*sz coefficients (SoA [64][sz][sy][sx])]
 *
 * Fit modes 0-5 keep the reference semantics (0 none, 1 Gaussian fixed sigma, 2 free sigma, 3 sigmaX/sigmaY,
 * 4 sigmaX/sigmaY/theta, 5 cubic spline EMCCD).
 *
 * Fit modes 6-8 are additions (the reference's fitRegions has no branch for them): Poisson maximum-likelihood fits of
 * (background, photons, x, y, s) on photon counts (ADU - offset) / gain, FP32 iterations, FP64 final pass.
 *   6 pixel-integrated Gaussian, s = sigma (px):  [roi, sigma0, offset, gain, maxIter, crlbMax]
 *   7 astigmatic Gaussian, s = z (nm):            [roi, pixelSize (nm), z0x, wx, c3x, c4x, Ax, z0y, wy, c3y, c4y, Ay,
 *                                                  offset, gain, maxIter, zMin, zMax, crlbMax]
 *     sigma_axis(z) = (A / pixelSize) sqrt(1 + u^2 + c3 u^3 + c4 u^4), u = (z - z0) / w (the AstigFit model)
 *   8 cubic spline, s = z (table cells):          [roi, sx, sy, sz, deltaZ, offset, gain, maxIter, crlbMax,
 *                                                  64*sx*sy*sz coefficients (SoA [64][sz][sy][sx])]
 * Their rows: X, Y, Z (nm; 0 for mode 6), Integrated intensity = photons, SigmaX/SigmaY (px; 0 for mode 8),
 * Theta = the FP64 Poisson deviance of the fit (-2 log of its likelihood ratio to the saturated model; a goodness of
 * fit), QualityXY = sqrt((CRLB_x^2 + CRLB_y^2) / 2) (px), QualityZ = CRLB_z (nm; -1 for mode 6), Amplitude, Offset =
 * background photons per pixel. A fit whose QualityXY exceeds crlbMax (when > 0) or that fails is a sentinel row
 * (-1 entries).
 *
 * Threading: every entry point may be called from several host threads at once (the reference is reentrant,
 * CPU/main.cpp:18-26). Each call leases an engine of the current device's pool - its own CUDA streams, device
 * workspace and launch-chain graphs - so concurrent calls run side by side on the GPU; a pool grows on demand up to
 * PTB_MAX_ENGINES engines per device (default 8), after which callers wait for a free engine. Results do not depend
 * on which engine ran a call.
 */
#ifndef PALMTRACER_B200_H
#define PALMTRACER_B200_H

#include <stdint.h>

#if defined(_WIN32)
#define PTB_API __declspec(dllexport)
#else
#define PTB_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces Localization (CPU/main.cpp:112-121): detection (a trous wavelet, threshold, watershed) and per-candidate
 * fit over a stack. Per-plane capacity is (outputSize / 18) / planes rows (lib/Palm.cpp:51); candidates beyond it
 * are dropped in label order with one stderr warning. Rows are sorted per plane by (Y, X) and numbered with a
 * global 1-based Id, the 1-based Plane and the per-plane 1-based Index. Returns the number of doubles written. */
PTB_API uint64_t Localization(const uint16_t* input, double* output, uint64_t outputSize, uint64_t height,
                              uint64_t width, uint64_t planes, double thresholdVal, double watershedRatio, uint64_t fit,
                              const double* fit_params);

/* Replaces Fitting (CPU/main.cpp:141-148 -> lib/Palm.cpp:73-119): fits at caller-given positions, rows in input
 * order, Id and Plane copied from the input, Index = rank within its plane. Returns nPoints * 18 (0 if empty). */
PTB_API uint64_t Fitting(const uint16_t* input, const double* positions, uint64_t nPoints, double* output,
                         uint64_t outputSize, uint64_t height, uint64_t width, uint64_t planes, uint64_t fit,
                         const double* fit_params);

/* Replaces Wavelett (CPU/main.cpp:257-284): one wavelet plane per frame as float64 [planes][height][width];
 * levelOutput is 1-based (0 is treated as 1) and clamped to the last plane (the residual). */
PTB_API void Wavelett(const uint16_t* input, double* output, uint64_t height, uint64_t width, uint64_t planes,
                      uint64_t levelOutput);

/* Replaces AutoThreshold (CPU/main.cpp:75-85 -> lib/Palm.cpp:122-172): iterative out-of-ROI standard deviation of
 * the raw pixels of frame 0 (at most 5 rounds of detection with fit 0 and watershed ratio 10). */
PTB_API double AutoThreshold(const uint16_t* input, uint64_t height, uint64_t width, const double* fit_params);

/* Replaces Astigmatism3DEstimation (CPU/main.cpp:324-353 -> lib/fit/AstigFit.cpp:36-72, 342-447): z of each point
 * from its fitted widths. input [size][2] = (sigma_x, sigma_y) in pixels, output [size][2] = (z in nm, compatibility
 * score in (0, 1]), model = [z0, w, c3, c4, A] of the x axis then of the y axis (nm), z searched in [-zMax, zMax]
 * (201-point grid, then Brent). Equals the reference bit for bit. */
PTB_API void Astigmatism3DEstimation(const double* input, double* output, uint64_t size, double pixelSize, const double* model,
                                     double zMax);

/* Replaces Tracking (CPU/main.cpp:159-164 -> lib/tracking/Tracks.cpp:69-212): links localizations of consecutive
 * planes greedily by increasing squared distance (pairs with dx^2 + dy^2 <= maxDistance^2, ties by source then target
 * in point order), then numbers the tracks 1, 2, ... from their first point. input [nPoints][4] = (Id, Plane, X, Y),
 * any order; output [nPoints][2] = (Id, Track) in (Plane, Id) order. Same results as the reference for distinct
 * (Plane, Id) pairs (equal pairs keep their input order). Writes nothing for nPoints = 0. */
PTB_API void Tracking(const double* input, uint64_t* output, uint64_t nPoints, double maxDistance);

/* Replaces the coefficient step of the spline calibration (lib/signal_processing/BSpline3D.cpp:17-164, run by
 * Spline::Calibrate at lib/signal_processing/Spline.cpp:52 on the averaged bead PSF with lambda = {0, 0, 100 / dz}):
 * the cubic smoothing-spline coefficient table of a PSF volume psf [nz][ny][nx] (x fastest; every dimension >= 2),
 * with regularisation lambda[3] per axis x, y, z (NULL: none, an interpolating spline). coeffs receives
 * 64 * (nx - 1) * (ny - 1) * (nz - 1) doubles in the layout the spline fits read, SoA [64][nz - 1][ny - 1][nx - 1]
 * (the reference emits [cell][64]): the table of fit_params for modes 5 and 8 with sx = nx - 1, sy = ny - 1,
 * sz = nz - 1. Returns the doubles written, 0 on error. */
PTB_API uint64_t PTB_SplineCoefficients(const double* psf, uint64_t nx, uint64_t ny, uint64_t nz, const double* lambda, double* coeffs);

/* ---- Additions (no counterpart in the reference) ---------------------------------------------------------------- */

/* Tracking on DEVICE buffers of the current CUDA device, ordered on `stream` (a cudaStream_t; the call synchronizes
 * it, since the plane range and the pair count size its scratch). Returns 2 * nPoints, or 0 on error. */
PTB_API uint64_t PTB_TrackingDevice(const double* d_input, uint64_t* d_output, uint64_t nPoints, double maxDistance, void* stream);

/* TIFF stacks (the reference's test-harness loader, Tests_CPU/TiffManagement.hpp:8-55, reads them with libtiff).
 * Multi-page, 16 bits and one sample per pixel, uncompressed strips, classic TIFF or BigTIFF in either byte order;
 * every page must have the first page's size (the reference's two checks). Host-only: no CUDA call.
 * PTB_TiffInfo: 1 and the stack's width, height and page count, or 0 (error in PTB_LastError()).
 * PTB_TiffRead: pages [first, first + count) into output ([count][height][width], host byte order); returns count,
 * or 0 on error. */
PTB_API int PTB_TiffInfo(const char* path, uint64_t* width, uint64_t* height, uint64_t* planes);
PTB_API uint64_t PTB_TiffRead(const char* path, uint16_t* output, uint64_t first, uint64_t count);

/* Localization of a TIFF stack on disk: same output, return value and parameters as Localization over the file's
 * pages. Chunk k + 1 is read from the file into pinned staging while chunk k computes on the GPU. */
PTB_API uint64_t PTB_LocalizationTiff(const char* path, double* output, uint64_t outputSize, double thresholdVal,
                                      double watershedRatio, uint64_t fit, const double* fit_params);

/* Same contract as Localization, but d_input and d_output are DEVICE memory of the current CUDA device (fit_params
 * stays a host array) and the work is ordered after the caller's `stream` (a cudaStream_t; 0 = legacy default
 * stream), which in turn waits for it. Blocks until the row count is known. Used when frames are already resident
 * in HBM (the serving and benchmark paths). */
PTB_API uint64_t PTB_LocalizationDevice(const uint16_t* d_input, double* d_output, uint64_t outputSize,
                                        uint64_t height, uint64_t width, uint64_t planes, double thresholdVal,
                                        double watershedRatio, uint64_t fit, const double* fit_params, void* stream);

/* Serving (additive surface; no counterpart in the reference). PTB_ServerStart starts `slots` worker slots on the
 * current device, each with its own CUDA stream and chunk workspace and an equal share of `budgetBytes` of device
 * memory (0 = half of the free memory); returns 1, or 0 on error. PTB_SubmitStack queues one Localization (same
 * arguments and output layout) and returns a ticket (0 on error); the input and output buffers stay owned by the
 * caller and must stay valid until the request completes (fit_params is copied). A queued stack starts when a slot is
 * free and its estimated device memory fits in what the running stacks leave of the budget (first fit in submission
 * order); stacks on different slots run concurrently on the device. Each result equals what Localization returns for
 * the same stack. PTB_PollStack: 0 queued or running, 1 done, -1 failed or unknown ticket. PTB_StackResult waits for
 * the request, releases the ticket and returns the doubles written (-1 on failure, message in PTB_LastError);
 * `times` (NULL or 2 doubles) receives the queueing delay and the latency from submission to completion in seconds.
 * PTB_ServerStop finishes the running stacks and fails the queued ones; call it with no other server call in flight.
 * Fit modes 6-8 are fused across requests: the slots hand each chunk's candidates to one fit stage, which waits a
 * short window (PTB_FUSE_WINDOW_US, default 300 us) for the chunks of the other busy slots and fits all chunks with
 * the same fit settings in ONE persistent launch over a shared device work queue, then scatters the rows back per
 * request (PTB_FUSE_FITS=0: each slot fits its own chunks). PTB_ServerFuseStats: counts[0] fused launches, counts[1]
 * chunks fitted by them, since the server started. */
PTB_API int PTB_ServerStart(int slots, uint64_t budgetBytes);
PTB_API uint64_t PTB_SubmitStack(const uint16_t* input, double* output, uint64_t outputSize, uint64_t height, uint64_t width,
                                 uint64_t planes, double thresholdVal, double watershedRatio, uint64_t fit, const double* fit_params);
PTB_API int PTB_PollStack(uint64_t ticket);
PTB_API int64_t PTB_StackResult(uint64_t ticket, double* times);
PTB_API void PTB_ServerStop(void);
PTB_API void PTB_ServerFuseStats(uint64_t* counts, int n);

/* Fit-only at caller-given positions with no device memory allocation: for callers that cannot call cudaMalloc
 * (code running inside another runtime's stream callbacks or under a fixed pre-sized memory pool) but can pass device
 * buffers. No counterpart in the reference; same result as Fitting for the same inputs. d_input is the device stack
 * uint16 [planes][height][width], d_positions the device rows [nPoints][6] (Id, Plane, X, Y, SegIntensity, Surface),
 * d_output the device rows [nPoints][18]; fit_params stays a host array. Work is enqueued on `stream` (cudaStream_t,
 * 0 = legacy default) and the call returns without waiting for it. Limits: at most 65536 points and 65536 planes,
 * fit modes 0-4, 6 and 7 (the spline modes need a device coefficient table); larger calls return 0 with an error.
 * Scratch lives in one static device array of about 3 MB that every GPU loading the library keeps until exit; it is
 * shared by all calls, so calls that overlap on the GPU race. The first call on a device looks up the array's device
 * address; make that first call before any stream capture. Returns nPoints * 18, or 0 (error or empty input). */
PTB_API uint64_t PTB_FittingDeviceNoAlloc(const uint16_t* d_input, const double* d_positions, uint64_t nPoints,
                                          double* d_output, uint64_t height, uint64_t width, uint64_t planes, uint64_t fit,
                                          const double* fit_params, void* stream);

/* Segmentation mode. Both modes give the reference's labels (Segmentation2D.cpp:336-385) for any threshold.
 * 0 (default): each 8-connected component of the thresholded potential is flooded on its own, in parallel, and then
 * tested: the flood of a component equals the reference's frame-wide flood when, at every basin boundary, the lowest
 * W1 along the winning parent chain exceeds the competing neighbour's W1 by more than the largest difference of aging
 * terms the frame-wide flood can give them. First test: the frame's domain pixel count x 1e-7 bounds that difference.
 * Boundaries failing it get the rank test, whose bound comes from the counts of the frame's pixels above and below
 * the two W1 levels (the frame-wide flood pops in W1 order up to the aging term). A frame failing the rank test is
 * flooded again per component with each pop's aging set to its estimated frame-wide position, and tested again with
 * per-element bounds; only a frame failing that too (or, with basin fusion, the rank test) is flooded again as one
 * unit with the frame-global pop counter. 1 (strict): every frame is flooded as one unit.
 * 2: as 0 with the first test only (every frame failing it is flooded again frame-wide; for comparisons).
 * Other values select 0. Returns the previous mode. */
PTB_API int PTB_SetSegmentationMode(int mode);

/* Segmentation diagnostics of the current device's engines since the last call: counts[0] frames segmented,
 * counts[1] frames flooded again frame-wide, counts[2] frames whose per-component floods needed the rank test (the
 * second exactness test) in mode 0, counts[3] frames flooded again per component with estimated frame-wide aging
 * after failing it, counts[4..10] the frames of counts[1] by the first reason they were flooded frame-wide: the list
 * of failing boundary pairs full, a pair failing the first test in mode 2, no rank-test slot left in the chunk, too
 * many failing pairs in the frame, a failed rank test after a basin fusion, no re-flood slot or too many domain
 * pixels for the re-flood, a failed re-flood test (up to n entries). */
PTB_API void PTB_SegmentationStats(uint64_t* counts, int n);

/* Engine pool of the current device (diagnostics): counts[0] engines created, counts[1] the most engines leased at
 * the same time (up to n entries). */
PTB_API void PTB_EnginePoolStats(uint64_t* counts, int n);

/* ROI mappings the autotuner chose for the maximum-likelihood modes 6-8 on the current device's engines
 * (diagnostics): up to n entries of 5 ints (mode, ROI size, chunk size class, lanes per ROI, work-queue chunk), one
 * per engine and tuned class. Returns the entries written. */
PTB_API int PTB_MleMappings(int* entries, int n);

/* Fit arithmetic for the Gaussian least-squares modes 1-4. 0 (default): FP64, one thread per ROI, in the
 * reference's exact order of operations (same iteration path as the reference); 1: FP32 iterations, one warp per
 * ROI, with an FP64 re-fit of every ROI whose FP32 run did not stop cleanly; 2: FP64, one warp per ROI.
 * Returns the previous setting. */
PTB_API int PTB_SetFitPrecision(int mode);

/* Last error message of the calling thread ("" when none). */
PTB_API const char* PTB_LastError(void);

/* Number of kernel launches issued by this library in the calling process so far (diagnostics). */
PTB_API uint64_t PTB_KernelLaunchCount(void);

/* Stage timing (diagnostics). When enabled, every chunk records CUDA events on the library's stream around its
 * stages and accumulates device milliseconds per stage: [0] detection kernel, [1] segmentation chain, [2] fit
 * kernels, [3] ordering and numbering, [4] host<->device copies, and for fit modes 6-8 the fit's phases: [5]
 * initial values, [6] Levenberg-Marquardt iterations, [7] Newton polish, [8] FP64 likelihood and CRLB (the
 * warp-per-ROI mapping runs as one launch, counted in [6]). PTB_StageTimes copies up to n totals into ms and the matching launch
 * counts into launches (either may be NULL), then resets them. Returns the previous setting. */
PTB_API int PTB_SetProfiling(int enable);
PTB_API void PTB_StageTimes(double* ms, uint64_t* launches, int n);

/* Model evaluations of fit modes 6-8 counted while profiling is enabled (diagnostics): [0] FP32 evaluations of the
 * Levenberg-Marquardt iterations, [1] FP32 evaluations of the Newton polish (with the rare Fisher-scoring fallbacks),
 * [2] evaluations of the initial axial pre-scan (FP32) and of the final Fisher information (FP64); one evaluation
 * visits every pixel of one ROI. [3] FP32 Cholesky
 * factorisations redone in FP64 (ill-conditioned or failed), counted always. Copies up to n totals into counts,
 * then resets them. */
PTB_API void PTB_MleEvaluations(uint64_t* counts, int n);

/* Launch-chain graphs of the current device's engines (diagnostics). A chunk's compute chain (counter reset,
 * detection, segmentation, candidates, fits) is launched directly the first time its launch arguments occur, captured
 * into a CUDA graph the second time and replayed from the graph after that (PTB_GRAPHS=0 turns graphs off).
 * counts: [chunks captured, chunks replayed, chunks launched directly] since the last call (up to n entries). */
PTB_API void PTB_GraphStats(uint64_t* counts, int n);

/* Input staging of the detection kernel (diagnostics, whole process): counts[0] = launches whose input tiles were
 * copied by the tensor memory accelerator (one bulk tensor copy per tile; frames whose width is a multiple of 8 in a
 * 16-byte aligned buffer, unless PTB_DETECT_TMA=0), counts[1] = launches staged with per-thread loads; launches issued
 * since the last call (a replay of a captured launch chain is not counted again), up to n entries. */
PTB_API void PTB_DetectStagingStats(uint64_t* counts, int n);

/* FMA throughput probe of the current device (diagnostics): FLOP/s (2 per FMA) of FP64 (fp64 != 0) or FP32
 * arithmetic, timed with CUDA events over a grid of independent FMA chains; -1 on error. */
PTB_API double PTB_MeasureFmaPeak(int fp64);

#ifdef __cplusplus
}
#endif

#endif /* PALMTRACER_B200_H */
