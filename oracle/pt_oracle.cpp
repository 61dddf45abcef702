// PALMTracer localization hot path: CPU restatement used as the ORACLE (test infrastructure only).
//
// Only tests/, the smoke check and the bench's CPU-baseline leg load this library, and only as the checker.
// The product (palmtracer-cpp_b200/) neither links nor calls anything here.
//
// Every function restates the reference algorithm (tmonseigne/PALMTracer-cpp 1.3.0) in FP64 with the same
// order of floating-point operations where the result depends on it, so that its outputs can be pinned
// BIT FOR BIT against the reference built from source (oracle/_ref) and against the reference's own golden
// CSVs (Tests_CPU/Input/ref/*.csv). Build flags follow the reference's strict mode (-ffp-contract=off).
//
// Entry points (extern "C", prefix orc_):
//   orc_Localization / orc_Fitting / orc_Wavelett / orc_AutoThreshold  - the four C-ABI exports
//   orc_Planes, orc_Candidates, orc_CandidatesFromPotential, orc_Labels - per-stage products
//   orc_Astig3DEstimation - z from (sigma_x, sigma_y) with the astigmatism model (the reference's export of that name)
//   orc_Tracking          - frame-to-frame linking (the reference's export of that name)
//   orc_SplineCoefficients - cubic-spline coefficient table of a PSF volume (spline calibration's BSpline3D step)
#include <omp.h>

#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <compare>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <numbers>
#include <queue>
#include <vector>

namespace {

// ---------------------------------------------------------------------------------------------
// Constants (lib/Constants.hpp:20-24, 53; lib/localization/Segmentation2D.hpp:80; lib/fit/Fitting.hpp:80)
constexpr int kPlaneId = 1;            // wavelet plane used for detection
constexpr int kNumPlanes = 3;          // detail planes W0, W1 and the residual V2
constexpr double kVolumeMin = 4;       // regions need surf > 4
constexpr int kThresholdIters = 5;     // AutoThreshold iterations
constexpr double kEps = 1e-7;          // EPSILON: watershed aging step and fill() guards
constexpr double kSeedFloor = 1e-8;    // Segmentation2D::THRESHOLD
constexpr int kMaxIter = 75;           // Fitting::N_ITER
constexpr int kCols = 18;              // localization_columns::Count

enum Col { cId = 0, cPlane, cIndex, cChannel, cX, cY, cZ, cIntensity, cSigmaX, cSigmaY, cTheta,
           cQualityXY, cQualityZ, cAmplitude, cOffset, cSegIntensity, cSurface, cCircularity };

// Fit modes (lib/fit/Fitting.hpp:22-30)
enum Mode { kNone = 0, kG2Fixed = 1, kG2Sigma = 2, kG3Fixed = 3, kG3Theta = 4, kSplineEmccd = 5 };

struct Candidate {  // lib/localization/SegmentationInfo.hpp:32-71 (only the fields that leave Segmentation2D)
	double x = 0, y = 0, z = 0, intensity = 0, surf = 0;
};

using Row = std::array<double, kCols>;

// ---------------------------------------------------------------------------------------------
// A trous B3 wavelet (lib/localization/ATrous.cpp:23-38, 49-80).
// V0 = image; V(k+1) = column pass of (row pass of Vk) with taps 3/8, 1/4, 1/16 at offsets 0, +-2^k, +-2^(k+1),
// each pass clamping its coordinate into the image; W(k) = Vk - V(k+1); the last plane keeps the residual.
void Atrous(const uint16_t* img, int H, int W, std::vector<double> planes[kNumPlanes])
{
	const size_t n = static_cast<size_t>(H) * W;
	for (int k = 0; k < kNumPlanes; ++k) { planes[k].assign(n, 0.0); }
	std::vector<double> tmp(n);
	for (size_t i = 0; i < n; ++i) { planes[0][i] = static_cast<double>(img[i]); }
	const double h0 = 3.0 / 8.0, h1 = 1.0 / 4.0, h2 = 1.0 / 16.0;
	auto cx = [W](int x) { return std::clamp(x, 0, W - 1); };
	auto cy = [H](int y) { return std::clamp(y, 0, H - 1); };
	for (int k = 0; k < kNumPlanes - 1; ++k) {
		const int s = 1 << k, s2 = 2 * s;
		const std::vector<double>& in = planes[k];
		std::vector<double>& out = planes[k + 1];
		for (int y = 0; y < H; ++y) {
			const double* r = in.data() + static_cast<size_t>(y) * W;
			for (int x = 0; x < W; ++x) {
				tmp[static_cast<size_t>(y) * W + x] = (h0 * r[x]) + (h1 * (r[cx(x - s)] + r[cx(x + s)])) + (h2 * (r[cx(x - s2)] + r[cx(x + s2)]));
			}
		}
		for (int y = 0; y < H; ++y) {
			for (int x = 0; x < W; ++x) {
				auto at = [&](int yy) { return tmp[static_cast<size_t>(cy(yy)) * W + x]; };
				out[static_cast<size_t>(y) * W + x] = (h0 * tmp[static_cast<size_t>(y) * W + x]) + (h1 * (at(y - s) + at(y + s))) + (h2 * (at(y - s2) + at(y + s2)));
			}
		}
		std::vector<double>& detail = planes[k];
		for (size_t i = 0; i < n; ++i) { detail[i] -= out[i]; }
	}
}

// ---------------------------------------------------------------------------------------------
// Segmentation (lib/localization/Segmentation2D.cpp).
struct Segmenter {
	int H = 0, W = 0;
	double ratio = 0;
	std::vector<double> pot;        // thresholded potential ("output_")
	std::vector<uint32_t> lab;      // label map ("map_")
	std::vector<Candidate> cands;   // per label ("infos_")

	size_t at(int y, int x) const { return static_cast<size_t>(y) * W + x; }

	// Strict threshold of plane 1 (Segmentation2D.cpp:50-74, comparison at :62).
	void Run(const double* plane1, int h, int w, double thr, double r)
	{
		H = h; W = w; ratio = r;
		const size_t n = static_cast<size_t>(H) * W;
		pot.assign(n, 0.0);
		lab.assign(n, 0);
		cands.clear();
		for (size_t i = 0; i < n; ++i) { pot[i] = plane1[i] > thr ? plane1[i] : 0.0; }
		Seeds();
		Flood();
		if (static_cast<int>(ratio) > 0) {  // WatershedIntelligent, Segmentation2D.cpp:77-85
			Fuse();
			Flood();
		}
		Statistics();
		Filter();
	}

	// Local maxima (Segmentation2D.cpp:294-333): v > 1e-8 and no 8-neighbour strictly greater. A maximum that touches an
	// already-labelled raster predecessor takes the first such label in 3x3 scan order; otherwise it opens a new label.
	void Seeds()
	{
		std::fill(lab.begin(), lab.end(), 0u);
		uint32_t next = 1;
		for (int i = 0; i < H; ++i) {
			for (int j = 0; j < W; ++j) {
				const double v = pot[at(i, j)];
				if (!(v > kSeedFloor)) { continue; }
				bool dominated = false;
				for (int ii = std::max(i - 1, 0); ii <= std::min(i + 1, H - 1) && !dominated; ++ii) {
					for (int jj = std::max(j - 1, 0); jj <= std::min(j + 1, W - 1) && !dominated; ++jj) {
						if ((ii != i || jj != j) && v < pot[at(ii, jj)]) { dominated = true; }
					}
				}
				if (dominated) { continue; }
				uint32_t inherit = 0;
				for (int ii = std::max(i - 1, 0); ii <= std::min(i + 1, H - 1) && inherit == 0; ++ii) {
					for (int jj = std::max(j - 1, 0); jj <= std::min(j + 1, W - 1) && inherit == 0; ++jj) {
						if ((ii != i || jj != j) && lab[at(ii, jj)] > 0) { inherit = lab[at(ii, jj)]; }
					}
				}
				lab[at(i, j)] = inherit > 0 ? inherit : next++;
			}
		}
		cands.assign(next - 1, Candidate{});
	}

	// Priority flood (Segmentation2D.cpp:336-385). Heap order is std::priority_queue with the reference's Pixel
	// comparison (lib/Structs.hpp:20-27: a < b iff a.v > b.v), so equal keys resolve exactly as in the reference.
	struct HeapPx {
		size_t x, y;  // x = row, y = column (reference naming)
		double v;
		bool operator<(const HeapPx& o) const { return v > o.v; }
	};

	void Flood()
	{
		std::priority_queue<HeapPx> heap;
		for (int x = 0; x < H; ++x) {
			for (int y = 0; y < W; ++y) {
				if (lab[at(x, y)] == 0) { continue; }
				bool open = false;
				for (int dx = -1; dx <= 1 && !open; ++dx) {
					const int nx = x + dx;
					if (nx < 0 || nx >= H) { continue; }
					for (int dy = -1; dy <= 1 && !open; ++dy) {
						const int ny = y + dy;
						if ((dx == 0 && dy == 0) || ny < 0 || ny >= W) { continue; }
						if (lab[at(nx, ny)] == 0) { open = true; }
					}
				}
				if (open) { heap.push(HeapPx{static_cast<size_t>(x), static_cast<size_t>(y), -pot[at(x, y)]}); }
			}
		}
		size_t pops = 0;
		while (!heap.empty()) {
			const HeapPx p = heap.top();
			heap.pop();
			++pops;
			for (int dx = -1; dx <= 1; ++dx) {
				const int nx = static_cast<int>(p.x) + dx;
				if (nx < 0 || nx >= H) { continue; }
				for (int dy = -1; dy <= 1; ++dy) {
					const int ny = static_cast<int>(p.y) + dy;
					if ((dx == 0 && dy == 0) || ny < 0 || ny >= W) { continue; }
					const size_t q = at(nx, ny);
					if (pot[q] > kSeedFloor && lab[q] == 0) {
						const double key = -pot[q] + (static_cast<double>(pops) * kEps);
						heap.push(HeapPx{static_cast<size_t>(nx), static_cast<size_t>(ny), key});
						lab[q] = lab[at(static_cast<int>(p.x), static_cast<int>(p.y))];
					}
				}
			}
		}
	}

	// Basin fusion (Segmentation2D.cpp:181-291): repeat until stable; a basin whose relative boundary contrast is below
	// `ratio` merges into its strongest-boundary neighbour when that neighbour peaks higher; one seed per basin remains.
	struct Basin {
		double maxWithNeighbour, minPot, maxPot;
		uint32_t row, col, neighbour, become, newIndex;
		bool locked;
	};

	void Fuse()
	{
		std::vector<Basin> b(cands.size());
		if (b.empty()) { return; }
		bool change = true;
		uint32_t count = 0;
		while (change) {
			change = false;
			for (size_t i = 0; i < b.size(); ++i) {
				b[i].maxWithNeighbour = -1e10;
				b[i].minPot = +1e10;
				b[i].maxPot = -1e10;
				b[i].neighbour = 0;
				b[i].locked = false;
				b[i].become = static_cast<uint32_t>(i);
				b[i].newIndex = 0;
			}
			for (int i = 0; i < H; ++i) {
				for (int j = 0; j < W; ++j) {
					const uint32_t s = lab[at(i, j)];
					if (s == 0) { continue; }
					Basin& r = b[s - 1];
					const double v = pot[at(i, j)];
					r.minPot = std::min(r.minPot, v);
					if (v > r.maxPot) {
						r.maxPot = v;
						r.row = static_cast<uint32_t>(i);
						r.col = static_cast<uint32_t>(j);
					}
					for (int ii = std::max(i - 1, 0); ii <= std::min(i + 1, H - 1); ++ii) {
						for (int jj = std::max(j - 1, 0); jj <= std::min(j + 1, W - 1); ++jj) {
							if (ii == i && jj == j) { continue; }
							const uint32_t ns = lab[at(ii, jj)];
							if (ns != 0 && ns != s && v > r.maxWithNeighbour) {
								r.maxWithNeighbour = v;
								r.neighbour = ns;
							}
						}
					}
				}
			}
			for (size_t i = 0; i < b.size(); ++i) {
				Basin& r = b[i];
				if (r.neighbour == 0) { continue; }
				const size_t ni = r.neighbour - 1;
				if (r.locked || b[ni].locked) { continue; }
				const double delta = r.maxPot - r.minPot;
				if (std::abs(delta) <= DBL_EPSILON) { continue; }
				if ((r.maxPot - r.maxWithNeighbour) / delta < ratio && r.maxPot < b[ni].maxPot) {
					r.become = static_cast<uint32_t>(ni);
					b[ni].locked = true;
					r.locked = true;
					change = true;
				}
			}
			count = 0;
			for (size_t i = 0; i < b.size(); ++i) { if (b[i].become == i) { b[i].newIndex = ++count; } }
			for (uint32_t& s : lab) { if (s != 0) { s = b[b[s - 1].become].newIndex; } }
			b.resize(count);
		}
		cands.assign(count, Candidate{});
		std::fill(lab.begin(), lab.end(), 0u);
		for (size_t i = 0; i < b.size(); ++i) {
			if (b[i].become == i) { lab[at(static_cast<int>(b[i].row), static_cast<int>(b[i].col))] = b[i].newIndex; }
		}
	}

	// Region statistics in raster order (Segmentation2D.cpp:144-175); only surf, intensity and the centroid leave.
	void Statistics()
	{
		std::vector<double> sum(cands.size(), 0.0);
		for (auto& c : cands) { c = Candidate{}; }
		for (int i = 0; i < H; ++i) {
			for (int j = 0; j < W; ++j) {
				const uint32_t s = lab[at(i, j)];
				if (s == 0) { continue; }
				Candidate& c = cands[s - 1];
				const double v = pot[at(i, j)];
				c.surf += 1;
				c.x += v * static_cast<double>(j);
				c.y += v * static_cast<double>(i);
				sum[s - 1] += v;
			}
		}
		for (size_t k = 0; k < cands.size(); ++k) {
			Candidate& c = cands[k];
			if (static_cast<int>(c.surf) == 0) { continue; }
			c.x /= sum[k];
			c.y /= sum[k];
			c.intensity = sum[k];
		}
	}

	// Keep regions with surf > VOLUME_MIN, in label order (Segmentation2D.cpp:88-141; filter table :20-39).
	void Filter()
	{
		std::vector<Candidate> kept;
		kept.reserve(cands.size());
		for (const auto& c : cands) { if (!(c.surf <= kVolumeMin)) { kept.push_back(c); } }
		cands.swap(kept);
	}
};

// ---------------------------------------------------------------------------------------------
// Gauss-Jordan inverse with row equilibration and partial pivoting (lib/signal_processing/Matrix.cpp:297-355).
// Returns false where the reference throws std::domain_error.
bool InvertGaussJordan(std::vector<double>& a, std::vector<double>& inv, int n)
{
	std::fill(inv.begin(), inv.end(), 0.0);
	for (int i = 0; i < n; ++i) {
		double scale = 0.0;
		for (int j = 0; j < n; ++j) {
			const double v = a[i * n + j];
			if (!std::isfinite(v)) { return false; }
			scale = std::max(scale, std::abs(v));
		}
		if (scale == 0.0) { return false; }
		for (int j = 0; j < n; ++j) { a[i * n + j] /= scale; }
		inv[i * n + i] = 1.0 / scale;
	}
	const double tol = std::numeric_limits<double>::epsilon() * static_cast<double>(n);
	for (int i = 0; i < n; ++i) {
		int piv = i;
		for (int j = i + 1; j < n; ++j) { if (std::abs(a[j * n + i]) > std::abs(a[piv * n + i])) { piv = j; } }
		if (!std::isfinite(a[piv * n + i]) || std::abs(a[piv * n + i]) <= tol) { return false; }
		if (piv != i) {
			for (int j = 0; j < n; ++j) {
				std::swap(a[i * n + j], a[piv * n + j]);
				std::swap(inv[i * n + j], inv[piv * n + j]);
			}
		}
		const double pinv = 1.0 / a[i * n + i];
		for (int j = 0; j < n; ++j) {
			a[i * n + j] *= pinv;
			inv[i * n + j] *= pinv;
		}
		for (int j = 0; j < n; ++j) {
			if (j == i) { continue; }
			const double f = a[j * n + i];
			for (int k = 0; k < n; ++k) {
				a[j * n + k] -= f * a[i * n + k];
				inv[j * n + k] -= f * inv[i * n + k];
			}
		}
	}
	for (double v : a) { if (!std::isfinite(v)) { return false; } }
	for (double v : inv) { if (!std::isfinite(v)) { return false; } }
	return true;
}

// ---------------------------------------------------------------------------------------------
// Output row fill (lib/fit/Fitting.cpp:61-106).
void FillRow(int mode, const Candidate& c, Row& r, double x, double y, double z, double offset = -1, double amp = -1,
             double sx = -1, double sy = -1, double theta = -1, double qxy = -1, double qz = -1)
{
	r[cId] = 0; r[cPlane] = 0; r[cIndex] = 0; r[cChannel] = -1;
	r[cX] = x; r[cY] = y; r[cZ] = z;
	if (mode == kNone) { r[cIntensity] = c.intensity; }
	else if (mode == kSplineEmccd) { r[cIntensity] = amp; }
	else { r[cIntensity] = (amp > kEps && sx > kEps && sy > kEps) ? 2.0 * std::numbers::pi * amp * sx * sy : -1; }
	r[cSigmaX] = sx; r[cSigmaY] = sy; r[cTheta] = theta;
	r[cQualityXY] = qxy; r[cQualityZ] = qz;
	r[cAmplitude] = amp; r[cOffset] = offset;
	r[cSegIntensity] = c.intensity; r[cSurface] = c.surf;
	r[cCircularity] = (sx > kEps && sy > kEps) ? std::min(sx, sy) / std::max(sx, sy) : 1;
}

// Shared per-fit configuration (lib/fit/Fitting.cpp:14-40; GaussianFit.cpp:39-45).
struct FitConfig {
	int mode = kNone, nParams = 4, roi = 0, half = 0, n = 0;
	double sigmaX = 1, sigmaY = 2, theta = 0;
	int W = 0, H = 0;
	const uint16_t* img = nullptr;

	void Init(int m, const double* fp, const uint16_t* image, int w, int h)
	{
		mode = m; img = image; W = w; H = h;
		switch (mode) {
			case kG2Sigma: nParams = 5; break;
			case kG3Fixed: nParams = 6; break;
			case kG3Theta: nParams = 7; break;
			case kSplineEmccd: nParams = 5; break;
			default: nParams = 4; break;
		}
		roi = static_cast<int>(static_cast<size_t>(fp[0]));
		if (mode >= kG2Fixed && mode <= kG3Theta) { sigmaX = fp[1]; sigmaY = fp[2]; theta = fp[3]; }
		if (roi % 2 == 0) { roi--; }
		half = roi / 2;
		n = roi * roi;
	}

	// ROI inside the image? (GaussianFit.cpp:51-56; unsigned comparisons as in the reference)
	bool Inside(size_t ux, size_t uy) const
	{
		const size_t h = static_cast<size_t>(half);
		return !(h > ux || ux >= static_cast<size_t>(W) - h || h > uy || uy >= static_cast<size_t>(H) - h);
	}
};

// Gaussian PSF value and gradient at offset (x, y) from the centre (lib/fit/GaussianModel.cpp:19-52).
struct GaussModel {
	double off, amp, sx, sy, sx2, sy2, c, s, c2, s2, cs;
	bool iso, hasSigma, hasTheta;

	static GaussModel Make(int mode, const double* p, double sigma, double theta)
	{
		GaussModel m{};
		m.off = p[0]; m.amp = p[1];
		if (mode == kG2Fixed || mode == kG2Sigma) {
			const double sg = mode == kG2Fixed ? sigma : p[4];
			m.sx = m.sy = sg; m.sx2 = m.sy2 = sg * sg;
			m.c = 1; m.s = 0; m.c2 = 1; m.s2 = 0; m.cs = 0;
			m.iso = true; m.hasSigma = mode == kG2Sigma; m.hasTheta = false;
		}
		else {
			const double th = mode == kG3Fixed ? theta : p[6];
			m.sx = p[4]; m.sy = p[5]; m.sx2 = p[4] * p[4]; m.sy2 = p[5] * p[5];
			m.c = std::cos(th); m.s = std::sin(th); m.c2 = m.c * m.c; m.s2 = m.s * m.s; m.cs = m.c * m.s;
			m.iso = false; m.hasSigma = false; m.hasTheta = mode == kG3Theta;
		}
		return m;
	}

	double Eval(double x, double y, double* g) const
	{
		const double X2 = x * x, Y2 = y * y;
		if (iso) {
			const double e = std::exp(-(X2 + Y2) / (2 * sx2));
			const double P = amp * e;
			if (g) {
				g[0] = 1; g[1] = e; g[2] = P * x / sx2; g[3] = P * y / sx2;
				if (hasSigma) { g[4] = P / (sx * sx2) * (X2 + Y2); }
			}
			return P + off;
		}
		const double xc = x * c, xs = x * s, yc = y * c, ys = y * s;
		const double f1 = (xc - ys) / sx, f2 = (xs + yc) / sy;
		const double e = std::exp(-((f1 * f1) + (f2 * f2)));
		const double P = amp * e;
		if (g) {
			const double xy = x * y, f3 = 2 * xy * cs, f4 = (2 * xy / sx2) - (2 * xy / sy2);
			g[0] = 1; g[1] = e;
			g[2] = P * (-(((-2 * c2 * x) + (2 * y * cs)) / sx2) - (((-2 * s2 * x) - (2 * y * cs)) / sy2));
			g[3] = P * ((((2 * s2 * y) - (2 * x * cs)) / sx2) - (((-2 * c2 * y) - (2 * x * cs)) / sy2));
			g[4] = P * (2 * ((xc * xc) - f3 + (ys * ys)) / (sx * sx2));
			g[5] = P * (2 * ((xs * xs) + f3 + (yc * yc)) / (sy * sy2));
			if (hasTheta) { g[6] = P * ((2 * cs * (((X2 - Y2) / sx2) + ((Y2 - X2) / sy2))) - (s2 * f4) + (c2 * f4)); }
		}
		return P + off;
	}
};

// Unweighted least-squares Levenberg-Marquardt (lib/fit/GaussianFit.cpp:48-295).
void FitGaussian(const FitConfig& cf, const Candidate& c, Row& out)
{
	const size_t ux = static_cast<size_t>(c.x), uy = static_cast<size_t>(c.y);
	if (!cf.Inside(ux, uy)) { FillRow(cf.mode, c, out, c.x, c.y, c.z); return; }
	const int np = cf.nParams, n = cf.n, h = cf.half;
	std::vector<double> gx(n), gy(n), gv(n), hat(n);
	double vmin = std::numeric_limits<double>::max(), vmax = std::numeric_limits<double>::lowest();
	for (int i = -h; i <= h; ++i) {  // ROI gather, Fitting.cpp:109-123
		for (int j = -h; j <= h; ++j) {
			const int k = (i + h) * cf.roi + (j + h);
			gx[k] = static_cast<double>(ux + j);
			gy[k] = static_cast<double>(uy + i);
			gv[k] = static_cast<double>(cf.img[(ux + j) + (uy + i) * static_cast<size_t>(cf.W)]);
			vmin = std::min(vmin, gv[k]);
			vmax = std::max(vmax, gv[k]);
		}
	}
	// Initial parameters and bounds (Fitting.cpp:126-175)
	double lo[7], p[7], hi[7];
	const double r2 = std::numbers::sqrt2_v<double>;
	lo[0] = 0; lo[1] = 0; lo[2] = c.x - 1; lo[3] = c.y - 1;
	p[0] = vmin; p[1] = vmax - vmin; p[2] = c.x; p[3] = c.y;
	hi[0] = 65535; hi[1] = 65535; hi[2] = c.x + 1; hi[3] = c.y + 1;
	if (cf.mode == kG2Sigma) { lo[4] = 0.1; p[4] = cf.sigmaX; hi[4] = 20; }
	if (cf.mode == kG3Fixed || cf.mode == kG3Theta) {
		lo[4] = lo[5] = 0.1; hi[4] = hi[5] = 20;
		p[4] = r2 * cf.sigmaX; p[5] = r2 * cf.sigmaY;
	}
	if (cf.mode == kG3Theta) { lo[6] = -150; p[6] = cf.theta; hi[6] = 150; }

	std::vector<double> alpha(np * np), alphaR(np * np), alphaRi(np * np);
	double beta[7], dp[7], pTry[7], grad[7];

	auto evalNormal = [&]() {  // GaussianFit.cpp:219-245
		std::fill(alpha.begin(), alpha.end(), 0.0);
		std::fill(beta, beta + np, 0.0);
		double err = 0.0;
		const GaussModel m = GaussModel::Make(cf.mode, p, cf.sigmaX, cf.theta);
		const bool circular = cf.mode == kG3Theta && std::abs(p[4] - p[5]) <= std::numeric_limits<double>::epsilon();
		for (int i = 0; i < n; ++i) {
			hat[i] = m.Eval(gx[i] - p[2], gy[i] - p[3], grad);
			const double d = gv[i] - hat[i];
			const double dw = 1.0 * d;
			err += d * dw;
			if (circular) { grad[6] = 0.0; }
			for (int a = 0; a < np; ++a) {
				beta[a] += grad[a] * dw;
				for (int b = 0; b < np; ++b) { alpha[a * np + b] += 1.0 * grad[a] * grad[b]; }
			}
		}
		return err;
	};
	auto trialError = [&]() {  // GaussianFit.cpp:262-271
		double res = 0.0;
		const GaussModel m = GaussModel::Make(cf.mode, pTry, cf.sigmaX, cf.theta);
		for (int i = 0; i < n; ++i) {
			const double d = gv[i] - m.Eval(gx[i] - pTry[2], gy[i] - pTry[3], nullptr);
			res += 1.0 * d * d;
		}
		return res;
	};
	auto maxAbsBeta = [&]() { double m = 0; for (int i = 0; i < np; ++i) { m = std::max(m, std::abs(beta[i])); } return m; };
	auto relStep = [&]() {
		double m = 0.0;
		for (int i = 0; i < np; ++i) { m = std::max(m, std::abs(dp[i]) / std::max(std::abs(p[i]), 1e-12)); }
		return m;
	};

	double err = evalNormal();
	bool finite = std::isfinite(err);
	for (int i = 0; i < np; ++i) { finite = finite && std::isfinite(beta[i]); }
	if (!finite) { FillRow(cf.mode, c, out, c.x, c.y, c.z); return; }
	double lambda = 1e-2;
	double m = maxAbsBeta();
	for (int it = (m < 1e-6) ? kMaxIter : 0; it < kMaxIter; ++it) {
		alphaR = alpha;
		for (int i = 0; i < np; ++i) {
			const int d = i * np + i;
			alphaR[d] = alpha[d] == 0.0 ? 1.0 : (1.0 + lambda) * alpha[d];
		}
		if (!InvertGaussJordan(alphaR, alphaRi, np)) {
			if (lambda < 1e7) { lambda = std::min(lambda * 11, 1e7); continue; }
			FillRow(cf.mode, c, out, c.x, c.y, c.z);
			return;
		}
		for (int i = 0; i < np; ++i) {
			dp[i] = 0.0;
			for (int j = 0; j < np; ++j) { dp[i] += alphaRi[i * np + j] * beta[j]; }
			if (!std::isfinite(dp[i])) { FillRow(cf.mode, c, out, c.x, c.y, c.z); return; }
			pTry[i] = std::clamp(p[i] + dp[i], lo[i], hi[i]);
		}
		for (int i = 0; i < np; ++i) { dp[i] = pTry[i] - p[i]; }
		bool tiny = true;
		for (int i = 0; i < np; ++i) { tiny &= (std::abs(dp[i]) < 1e-15); }
		if (tiny) {
			if (lambda >= 1e7) { break; }
			lambda = std::min(lambda * 11, 1e7);
			continue;
		}
		double quad = 0.0, lin = 0.0;  // predicted gain, GaussianFit.cpp:248-259
		for (int i = 0; i < np; ++i) {
			double t = 0.0;
			for (int j = 0; j < np; ++j) { t += alpha[i * np + j] * dp[j]; }
			quad += dp[i] * t;
			lin += dp[i] * beta[i];
		}
		const double gain = (2.0 * lin) - quad;
		if (gain <= 0.0) {
			if (lambda >= 1e7) { break; }
			lambda = std::min(lambda * 11, 1e7);
			if (relStep() < 1e-6 && it >= 2) { break; }
			continue;
		}
		double denom = 0.0;
		for (int i = 0; i < np; ++i) { denom += dp[i] * ((lambda * dp[i]) + beta[i]); }
		const double errTry = trialError();
		const double rho = (err - errTry) / (2.0 * denom);
		if (rho > 1e-2) {
			for (int i = 0; i < np; ++i) { p[i] = pTry[i]; }
			err = evalNormal();
			lambda = std::max(lambda / 9, 1e-7);
		}
		else {
			if (lambda >= 1e7) { break; }
			lambda = std::min(lambda * 11, 1e7);
		}
		if (it >= 2) {
			if (relStep() < 1e-6) { break; }
			if (err / static_cast<double>(n) < 1e-5) { break; }
			if (maxAbsBeta() < 1e-6) { break; }
		}
	}
	const double offset = p[0], amp = p[1], x = p[2], y = p[3];
	// Squared correlation of data and model (GaussianFit.cpp:274-295)
	double muD = 0.0, muM = 0.0;
	for (int i = 0; i < n; ++i) { muD += gv[i]; }
	for (int i = 0; i < n; ++i) { muM += hat[i]; }
	muD /= static_cast<double>(n);
	muM /= static_cast<double>(n);
	double t1 = 0.0, t2 = 0.0, t3 = 0.0;
	for (int i = 0; i < n; ++i) { t1 += (gv[i] - muD) * (hat[i] - muM); }
	for (int i = 0; i < n; ++i) { t2 += (gv[i] - muD) * (gv[i] - muD); }
	for (int i = 0; i < n; ++i) { t3 += (hat[i] - muM) * (hat[i] - muM); }
	const double R = t1 / std::sqrt(t2 * t3);
	const double r2score = std::isnan(R) ? 0 : R * R;
	if (r2score < kEps) { FillRow(cf.mode, c, out, x, y, c.z); return; }
	double sx = cf.sigmaX, sy = cf.sigmaY, th = cf.theta;
	switch (cf.mode) {
		case kG2Fixed: sx = sy = cf.sigmaX; th = 0; break;
		case kG2Sigma: sx = p[4]; sy = sx; th = 0; break;
		case kG3Fixed: sx = p[4] / r2; sy = p[5] / r2; break;
		case kG3Theta: sx = p[4] / r2; sy = p[5] / r2; th = p[6]; break;
		default: break;
	}
	FillRow(cf.mode, c, out, x, y, c.z, offset, amp, sx, sy, th, r2score);
}

// ---------------------------------------------------------------------------------------------
// Cubic-spline PSF Poisson LM, EMCCD (lib/fit/SplineFit.cpp:36-318).
struct SplineTable {
	int roi = 0, half = 0, n = 0, sx = 0, sy = 0, sz = 0;
	size_t sizeXY = 0, size = 0, offsetXY = 0;
	double initZ = 0, deltaZ = 0, intensityRatio = 1;
	const double* coeffs = nullptr;  // SoA [64][sz][sy][sx]

	void Init(const double* fp)
	{
		roi = static_cast<int>(static_cast<size_t>(fp[0]));
		sx = static_cast<int>(static_cast<size_t>(fp[1]));
		sy = static_cast<int>(static_cast<size_t>(fp[2]));
		sz = static_cast<int>(static_cast<size_t>(fp[3]));
		deltaZ = fp[4];
		coeffs = fp + 5;
		sizeXY = static_cast<size_t>(sx) * sy;
		size = sizeXY * sz;
		initZ = static_cast<double>(sz) / 2.0;
		const double centre = coeffs[(32 * size) + (sz / 2 * sizeXY) + (sy / 2 * static_cast<size_t>(sx)) + (sx / 2)];
		intensityRatio = std::abs(centre) < std::numeric_limits<double>::epsilon() ? 1.0 : 4.0 / centre;
		const int roiParsed = roi;
		offsetXY = static_cast<size_t>(std::floor((static_cast<double>(sx) + 1.0 - static_cast<double>(roiParsed)) / 2));
		if (roi % 2 == 0) { roi--; }
		half = roi / 2;
		n = roi * roi;
	}
};

// Monomial patch weights f = x^k y^j z^i and their derivatives (SplineFit.cpp:296-318).
void PatchWeights(double x, double y, double z, double f[64], double dfx[64], double dfy[64], double dfz[64])
{
	for (int i = 0; i < 64; ++i) { f[i] = dfx[i] = dfy[i] = dfz[i] = 0; }
	double cz = 1.0;
	for (int i = 0; i < 4; ++i) {
		double cy = 1.0;
		for (int j = 0; j < 4; ++j) {
			double cx = 1.0;
			for (int k = 0; k < 4; ++k) {
				const int id = i * 16 + j * 4 + k;
				const double w = cz * cy * cx;
				f[id] = w;
				if (k + 1 < 4) { dfx[id + 1] = static_cast<double>(k + 1) * w; }
				if (j + 1 < 4) { dfy[id + 4] = static_cast<double>(j + 1) * w; }
				if (i + 1 < 4) { dfz[id + 16] = static_cast<double>(i + 1) * w; }
				cx *= x;
			}
			cy *= y;
		}
		cz *= z;
	}
}

// Model value and derivatives at one spline cell (SplineFit.cpp:219-240); the cell is clamped into the table.
void SplineEval(const SplineTable& t, long px, long py, long pz, const double f[64], const double dfx[64], const double dfy[64],
                const double dfz[64], const double* p, double dudt[5], double& model)
{
	// Vec3I::Clamp with size_t arithmetic: a negative index wraps to a huge value and clamps to the upper bound.
	auto clampU = [](long v, int dim) {
		const size_t u = static_cast<size_t>(v);
		return std::min<size_t>(u, static_cast<size_t>(dim - 1));
	};
	const size_t x = clampU(px, t.sx), y = clampU(py, t.sy), z = clampU(pz, t.sz);
	const size_t pos = ((z * t.sy) + y) * t.sx + x;
	for (int i = 0; i < 5; ++i) { dudt[i] = 0.0; }
	for (int i = 0; i < 64; ++i) {
		const double cval = t.coeffs[i * t.size + pos];
		dudt[1] += f[i] * cval;
		dudt[2] += dfx[i] * cval;
		dudt[3] += dfy[i] * cval;
		dudt[4] += dfz[i] * cval;
	}
	dudt[0] = 1;
	dudt[2] *= -1 * p[1];
	dudt[3] *= -1 * p[1];
	dudt[4] *= p[1];
	model = p[0] + (p[1] * dudt[1]);
}

// Cholesky as in lib/signal_processing/Matrix.cpp:272-294 (l holds the transpose of u).
bool Cholesky(const double* a, int n, double* l, double* u)
{
	for (int i = 0; i < n; ++i) {
		for (int j = 0; j < i + 1; ++j) {
			double s = 0;
			for (int k = 0; k < j; ++k) { s += u[i * n + k] * u[j * n + k]; }
			if (i == j) {
				if (a[i * n + i] - s >= 0) {
					u[i * n + j] = std::sqrt(a[i * n + i] - s);
					l[j * n + i] = u[i * n + j];
				}
				else { return false; }
			}
			else {
				u[i * n + j] = 1.0 / u[j * n + j] * (a[i * n + j] - s);
				l[j * n + i] = u[i * n + j];
			}
		}
	}
	return true;
}

// In-place LU inverse without pivoting (lib/signal_processing/Matrix.cpp:358-410), column-major indexing as there.
void InverseLU(double* in, double* out, int n)
{
	std::vector<double> y(static_cast<size_t>(n) * n);
	double acc = 0;
	for (int j = 0; j < n; ++j) {
		for (int i = 0; i <= j; ++i) {
			if (i > 0) {
				for (int k = 0; k <= i - 1; ++k) { acc += in[i + (k * n)] * in[k + (j * n)]; }
				in[i + (j * n)] -= acc;
				acc = 0;
			}
		}
		for (int i = j + 1; i < n; ++i) {
			if (j > 0) {
				for (int k = 0; k <= j - 1; ++k) { acc += in[i + (k * n)] * in[k + (j * n)]; }
				in[i + (j * n)] = (1 / in[j + (j * n)]) * (in[i + (j * n)] - acc);
				acc = 0;
			}
			else { in[i + (j * n)] = (1 / in[j + (j * n)]) * in[i + (j * n)]; }
		}
	}
	for (int num = 0; num < n; ++num) {
		y[0] = num == 0 ? 1 : 0;
		for (int i = 1; i < n; ++i) {
			const size_t b = i == num ? 1 : 0;
			for (int j = 0; j <= i - 1; ++j) { acc += in[i + (j * n)] * y[j]; }
			y[i] = static_cast<double>(b) - acc;
			acc = 0;
		}
		out[n - 1 + (num * n)] = y[n - 1] / in[(n - 1) + ((n - 1) * n)];
		for (int i = n - 2; i >= 0; --i) {
			for (int j = i + 1; j < n; ++j) { acc += in[i + (j * n)] * out[j + (num * n)]; }
			out[i + (num * n)] = (1 / in[i + (i * n)]) * (y[i] - acc);
			acc = 0;
		}
	}
}

// Spline fit (SplineFit.cpp:53-216). Its bounds use the raw fitParams[0] (the ROI before it is forced odd).
void FitSplineFull(const SplineTable& t, double roiParam, const uint16_t* img, int W, int H, const Candidate& c, Row& out)
{
	constexpr int np = 5;
	const size_t ux = static_cast<size_t>(c.x), uy = static_cast<size_t>(c.y);
	const size_t h = static_cast<size_t>(t.half);
	if (h > ux || ux >= static_cast<size_t>(W) - h || h > uy || uy >= static_cast<size_t>(H) - h) {
		FillRow(kSplineEmccd, c, out, c.x, c.y, c.z);
		return;
	}
	const int n = t.n, roi = t.roi, hh = t.half;
	std::vector<double> gv(n);
	double vmin = std::numeric_limits<double>::max(), vmax = std::numeric_limits<double>::lowest();
	for (int i = -hh; i <= hh; ++i) {
		for (int j = -hh; j <= hh; ++j) {
			const int k = (i + hh) * roi + (j + hh);
			gv[k] = static_cast<double>(img[(ux + j) + (uy + i) * static_cast<size_t>(W)]);
			vmin = std::min(vmin, gv[k]);
			vmax = std::max(vmax, gv[k]);
		}
	}
	double x = 0, y = 0, sum = 0;
	for (int i = 0, k = 0; i < roi; ++i) {
		for (int j = 0; j < roi; ++j, ++k) {
			y += gv[k] * static_cast<double>(i);
			x += gv[k] * static_cast<double>(j);
			sum += gv[k];
		}
	}
	if (sum > 0) { x /= sum; y /= sum; }
	else { x = static_cast<double>(roi) / 2.0; y = static_cast<double>(roi) / 2.0; }
	const double roiC = (roiParam - 1) / 2.0, roiD = roiParam / 4.0;
	const double dmin = roiC - roiD, dmax = roiC + roiD;
	double lo[np] = {-0.01, -1, dmin, dmin, 0};
	double p[np] = {vmin, vmax - vmin, x, y, t.initZ};
	double hi[np] = {0.01, 1, dmax, dmax, 1};
	p[1] *= t.intensityRatio;
	hi[4] = static_cast<double>(t.sz);
	for (int i = 0; i < np; ++i) { p[i] = std::clamp(p[i], lo[i], hi[i]); }
	double jump[np] = {std::max(20.0, p[1]), std::max(100.0, p[1]), 1.0, 1.0, std::max(static_cast<double>(t.sz) / 3.0, 2.0)};

	double lambda = 0.1, err = std::numeric_limits<double>::max(), mu = 1 + lambda, model = 0;
	double hess[np * np], l[np * np], u[np * np], jac[np], upd[np] = {0, 0, 0, 0, 0}, dudt[np];
	double f[64], dfx[64], dfy[64], dfz[64];
	auto cellOrigin = [&](const double* pp, long& xi, long& yi, long& zi, double& xc, double& yc, double& zc) {
		const double xr = -1 * (pp[2] - static_cast<double>(hh) + 0.5), yr = -1 * (pp[3] - static_cast<double>(hh) + 0.5);
		xi = static_cast<int>(std::floor(xr));
		yi = static_cast<int>(std::floor(yr));
		zi = static_cast<int>(std::floor(pp[4]));
		xc = xr - static_cast<double>(xi);
		yc = yr - static_cast<double>(yi);
		zc = pp[4] - static_cast<double>(zi);
	};
	auto upMu = [&](bool up) {  // SplineFit.cpp:263-273
		if (up) { mu = std::max((1 + (lambda * 10)) / (1 + lambda), 1.3); lambda = 10 * lambda; }
		else { lambda = 0.1 * lambda; mu = 1 + lambda; }
	};
	bool stop = false;
	int it = 0;
	while (!stop) {
		++it;
		const double oldErr = err;
		double oldP[np], oldUpd[np];
		std::copy(p, p + np, oldP);
		std::copy(upd, upd + np, oldUpd);
		const double oldLambda = lambda;
		std::fill(jac, jac + np, 0.0);
		std::fill(hess, hess + np * np, 0.0);
		std::fill(upd, upd + np, 0.0);
		std::fill(l, l + np * np, 0.0);
		std::fill(u, u + np * np, 0.0);
		long xi, yi, zi;
		double xc, yc, zc;
		cellOrigin(p, xi, yi, zi, xc, yc, zc);
		PatchWeights(xc, yc, zc, f, dfx, dfy, dfz);
		for (int i = 0, k = 0; i < roi; ++i) {
			const long cx = xi + i + static_cast<long>(t.offsetXY);
			for (int j = 0; j < roi; ++j, ++k) {
				const long cy = yi + j + static_cast<long>(t.offsetXY);
				SplineEval(t, cx, cy, zi, f, dfx, dfy, dfz, p, dudt, model);
				const double d = gv[k];
				if (d > 0) { err = err + (2 * (model - d - (d * std::log(model / d)))); }
				else { err = err + (2 * model); }
				const double t1 = 1 - (d / model);
				for (int a = 0; a < np; ++a) { jac[a] += t1 * dudt[a]; }
				const double t2 = d / (model * model);
				for (int a = 0; a < np; ++a) {
					for (int b = a; b < np; ++b) {
						hess[a * np + b] += t2 * dudt[a] * dudt[b];
						hess[b * np + a] = hess[a * np + b];
					}
				}
			}
		}
		for (int a = 0; a < np; ++a) { hess[a * np + a] = hess[a * np + a] * mu; }
		if (Cholesky(hess, np, l, u)) {
			double yv[np];  // forward then backward substitution (SplineFit.cpp:276-294)
			for (int a = 0; a < np; ++a) {
				yv[a] = jac[a];
				for (int b = 0; b < a; ++b) { yv[a] -= l[b * np + a] * yv[b]; }
				yv[a] /= l[a * np + a];
			}
			for (int a = np - 1; a >= 0; --a) {
				upd[a] = yv[a];
				for (int b = a + 1; b < np; ++b) { upd[a] -= u[b * np + a] * upd[b]; }
				upd[a] /= u[a * np + a];
			}
			for (int a = 0; a < np; ++a) {
				if (std::abs(oldUpd[a]) > kEps && upd[a] / oldUpd[a] < -0.5) { jump[a] *= 0.5; }
				const double scale = upd[a] / (1.0 + (std::abs(upd[a]) / jump[a]));
				p[a] -= scale;
				p[a] = std::clamp(p[a], lo[a], hi[a]);
				upd[a] = scale;
			}
			if (err > oldErr) {
				err = oldErr;
				std::copy(oldP, oldP + np, p);
				std::copy(oldUpd, oldUpd + np, upd);
				lambda = oldLambda;
				upMu(true);
			}
			else { upMu(false); }
		}
		else {
			err = oldErr;
			std::copy(oldP, oldP + np, p);
			std::copy(oldUpd, oldUpd + np, upd);
			lambda = oldLambda;
			upMu(true);
		}
		if (it >= kMaxIter) { stop = true; }
		if (it > 2 && (err < 1e-6 || std::abs(err - oldErr) / err < 1e-6)) { stop = true; }
	}
	// CRLB (SplineFit.cpp:164-205)
	double fm[np * np] = {}, fmi[np * np] = {}, crlb[np];
	{
		long xi, yi, zi;
		double xc, yc, zc;
		cellOrigin(p, xi, yi, zi, xc, yc, zc);
		PatchWeights(xc, yc, zc, f, dfx, dfy, dfz);
		for (int i = 0; i < roi; ++i) {
			const long cx = xi + i + static_cast<long>(t.offsetXY);
			for (int j = 0; j < roi; ++j) {
				const long cy = yi + j + static_cast<long>(t.offsetXY);
				SplineEval(t, cx, cy, zi, f, dfx, dfy, dfz, p, dudt, model);
				for (int a = 0; a < np; ++a) {
					for (int b = a; b < np; ++b) {
						fm[a * np + b] += dudt[b] * dudt[a] / model;
						fm[b * np + a] = fm[a * np + b];
					}
				}
			}
		}
	}
	for (int a = 0; a < np; ++a) {
		if (std::abs(fm[a * np + a]) < std::numeric_limits<double>::epsilon()) { fm[a * np + a] = 1e-10; }
	}
	InverseLU(fm, fmi, np);
	for (int a = 0; a < np; ++a) { const double v = fmi[a * np + a]; crlb[a] = std::isnan(v) ? v : (v >= 0 ? std::sqrt(v) : 0.0); }
	const double off = crlb[0], amp = crlb[1], qxy = (crlb[2] + crlb[3]) / 2, qz = t.deltaZ * crlb[4];
	const double xo = p[2] - static_cast<double>(hh) + c.x;
	const double yo = p[3] - static_cast<double>(hh) + c.y;
	const double zo = t.deltaZ * (p[4] - t.initZ);
	FillRow(kSplineEmccd, c, out, xo, yo, zo, off, amp, 0, 0, 0, qxy, qz);
}

}  // namespace

// =============================================================================================================
// Maximum-likelihood fits (modes 6, 7, 8). These have no counterpart in the reference: they follow the benchmark
// workloads' definition (Poisson MLE of x, y, I, bg and sigma or z on camera data converted to photons) and are
// restated here in FP64 from the model maths as the oracle of the GPU modes. Parity for them is pinned by this
// restatement and by synthetic ground truth, not by the reference.
//
// Model: mu_k = bg + I * PSF(pixel k; x, y, s). Mode 6: PSF = Ex(x, sigma) Ey(y, sigma) with Ex the Gaussian
// integrated over the pixel, Ex = (erf(b) - erf(a)) / 2, a = (c - x - 1/2) / (sqrt2 sigma), b = (c - x + 1/2) /
// (sqrt2 sigma). Mode 7: sigma_x(z), sigma_y(z) from the astigmatism model of lib/fit/AstigFit.cpp:76-88
// (sigma_px = A / pixelSize * sqrt(max(0, 1 + U^2 + c3 U^3 + c4 U^4)), U = (z - z0) / w, coefficients per axis in
// the order [z0, w, c3, c4, A]). Mode 8: PSF = the cubic-spline table of SplineFit (monomial weights per cell), with
// the PSF centre at table coordinates ((sx - 1) / 2, (sy - 1) / 2) and z_nm = deltaZ * (Z - sz / 2).
// Objective: Poisson deviance D = 2 sum(mu - d - d ln(mu / d)); damped Fisher scoring (Levenberg-Marquardt with
// H = 2 sum mu^-1 dmu dmu^T) until the step is small; then FP64 Newton steps on the exact Hessian of the deviance to
// a 1e-10 relative step, both holding parameters on active bounds (FixActive); the CRLB sqrt(diag(F^-1)) from the FP64 Fisher information F = sum mu^-1 dmu dmu^T.
namespace {

struct MleCfg {
	int model = 6, roi = 7, half = 3, n = 49, maxIter = 20;
	double sigma0 = 1.3, offset = 100, gain = 2, crlbMax = 0;
	double pixelSize = 160, astig[10] = {}, zMin = -800, zMax = 800;
	int sx = 0, sy = 0, sz = 0;
	double dz = 10;
	const double* coeffs = nullptr;  // SoA [64][sz][sy][sx]
	size_t cells = 0;
};

bool ParseMle(int mode, const double* fp, MleCfg& c)
{
	c.model = mode;
	int roi = static_cast<int>(static_cast<size_t>(fp[0]));
	if (mode == 6) {
		c.sigma0 = fp[1]; c.offset = fp[2]; c.gain = fp[3]; c.maxIter = static_cast<int>(fp[4]); c.crlbMax = fp[5];
	}
	else if (mode == 7) {
		c.pixelSize = fp[1];
		for (int i = 0; i < 10; ++i) { c.astig[i] = fp[2 + i]; }
		c.offset = fp[12]; c.gain = fp[13]; c.maxIter = static_cast<int>(fp[14]); c.zMin = fp[15]; c.zMax = fp[16];
		c.crlbMax = fp[17];
	}
	else {
		c.sx = static_cast<int>(fp[1]); c.sy = static_cast<int>(fp[2]); c.sz = static_cast<int>(fp[3]); c.dz = fp[4];
		c.offset = fp[5]; c.gain = fp[6]; c.maxIter = static_cast<int>(fp[7]); c.crlbMax = fp[8];
		c.coeffs = fp + 9;
		c.cells = static_cast<size_t>(c.sx) * c.sy * c.sz;
	}
	if (roi % 2 == 0) { roi--; }
	c.roi = roi; c.half = roi / 2; c.n = roi * roi;
	return roi >= 1 && c.gain > 0;
}

// Pixel-integrated 1D Gaussian E(x, s) = (erf(b) - erf(a)) / 2, a = (c - x - 1/2) / (sqrt2 s), b = (c - x + 1/2) /
// (sqrt2 s), with its first derivatives (position, width) and, when d2 is given, the second derivatives
// d2 = {E_xx, E_xs, E_ss}.
void Erf1D(double c, double x, double s, double& e, double& dx, double& ds, double* d2 = nullptr)
{
	const double k = 1.0 / (1.4142135623730951 * s);
	const double a = (c - x - 0.5) * k, b = (c - x + 0.5) * k;
	const double ea = std::exp(-a * a), eb = std::exp(-b * b);
	e = 0.5 * (std::erf(b) - std::erf(a));
	dx = (ea - eb) / (2.5066282746310002 * s);
	ds = (a * ea - b * eb) / (1.7724538509055160 * s);
	if (d2) {
		d2[0] = (a * ea - b * eb) / (1.7724538509055160 * s * s);
		d2[1] = (2 * a * a * ea - 2 * b * b * eb - ea + eb) / (2.5066282746310002 * s * s);
		d2[2] = 2 * (a * (a * a - 1) * ea - b * (b * b - 1) * eb) / (1.7724538509055160 * s * s);
	}
}

// Astigmatic width (pixels), d width / dz and d2 width / dz2 for one axis [z0, w, c3, c4, A].
void AstigSigma(const double* m, double pixelSize, double z, double& s, double& ds, double* dss = nullptr)
{
	const double u = (z - m[0]) / m[1];
	const double poly = 1.0 + u * u + m[2] * u * u * u + m[3] * u * u * u * u;
	const double k = m[4] / pixelSize;
	if (poly <= 1e-12) { s = k * 1e-6; ds = 0; if (dss) { *dss = 0; } return; }
	const double r = std::sqrt(poly);
	const double p1 = 2 * u + 3 * m[2] * u * u + 4 * m[3] * u * u * u;
	const double p2 = 2 + 6 * m[2] * u + 12 * m[3] * u * u;
	s = k * r;
	ds = k * p1 / (2 * r * m[1]);
	if (dss) { *dss = k / (m[1] * m[1]) * (p2 / (2 * r) - p1 * p1 / (4 * r * poly)); }
}

// Spline PSF value and gradient at table coordinates (X, Y, Z); with h2 the second derivatives
// {S_XX, S_XY, S_XZ, S_YY, S_YZ, S_ZZ}.
double SplinePsf(const MleCfg& c, double X, double Y, double Z, double& dX, double& dY, double& dZ, double* h2 = nullptr)
{
	auto cell = [](double v, int dim, double& frac) {
		int i = static_cast<int>(std::floor(v));
		i = std::min(std::max(i, 0), dim - 1);
		frac = v - static_cast<double>(i);
		return i;
	};
	double fx, fy, fz;
	const int ix = cell(X, c.sx, fx), iy = cell(Y, c.sy, fy), iz = cell(Z, c.sz, fz);
	const size_t pos = (static_cast<size_t>(iz) * c.sy + iy) * c.sx + ix;
	double px[4] = {1, fx, fx * fx, fx * fx * fx}, py[4] = {1, fy, fy * fy, fy * fy * fy}, pz[4] = {1, fz, fz * fz, fz * fz * fz};
	double dpx[4] = {0, 1, 2 * fx, 3 * fx * fx}, dpy[4] = {0, 1, 2 * fy, 3 * fy * fy}, dpz[4] = {0, 1, 2 * fz, 3 * fz * fz};
	const double ddpx[4] = {0, 0, 2, 6 * fx}, ddpy[4] = {0, 0, 2, 6 * fy}, ddpz[4] = {0, 0, 2, 6 * fz};
	double v = 0;
	dX = dY = dZ = 0;
	if (h2) { for (int q = 0; q < 6; ++q) { h2[q] = 0; } }
	for (int i = 0; i < 4; ++i) {
		for (int j = 0; j < 4; ++j) {
			for (int m = 0; m < 4; ++m) {
				const double co = c.coeffs[static_cast<size_t>(i * 16 + j * 4 + m) * c.cells + pos];
				v += co * pz[i] * py[j] * px[m];
				dX += co * pz[i] * py[j] * dpx[m];
				dY += co * pz[i] * dpy[j] * px[m];
				dZ += co * dpz[i] * py[j] * px[m];
				if (h2) {
					h2[0] += co * pz[i] * py[j] * ddpx[m];
					h2[1] += co * pz[i] * dpy[j] * dpx[m];
					h2[2] += co * dpz[i] * py[j] * dpx[m];
					h2[3] += co * pz[i] * ddpy[j] * px[m];
					h2[4] += co * dpz[i] * dpy[j] * px[m];
					h2[5] += co * ddpz[i] * py[j] * px[m];
				}
			}
		}
	}
	return v;
}

struct MleRoi {
	const MleCfg* c;
	std::vector<double> d;  // photons, row-major
	double x0, y0;          // local candidate position

	// mu, dmu/dtheta (g, 5 per pixel) and, when h is given, d2mu/dtheta2 (upper triangle, 15 per pixel) for
	// theta = [bg, I, x, y, s].
	void Eval(const double* t, std::vector<double>& mu, std::vector<double>& g, std::vector<double>* h = nullptr) const
	{
		const MleCfg& C = *c;
		const int roi = C.roi, hh = C.half;
		mu.assign(C.n, 0);
		g.assign(static_cast<size_t>(C.n) * 5, 0);
		if (h) { h->assign(static_cast<size_t>(C.n) * 15, 0); }
		auto put2 = [&](int k, double Pxx, double Pxy, double Pxs, double Pyy, double Pys, double Pss, double Px, double Py, double Ps) {
			// d2mu: (I,x) = Px, (I,y) = Py, (I,s) = Ps, (x,x) = I Pxx, ... ; bg row and (I,I) are zero
			double* q = h->data() + static_cast<size_t>(k) * 15;
			const double I = t[1];
			// packed order: (0,0..4) (1,1..4) (2,2..4) (3,3..4) (4,4)
			q[0] = q[1] = q[2] = q[3] = q[4] = 0;
			q[5] = 0; q[6] = Px; q[7] = Py; q[8] = Ps;
			q[9] = I * Pxx; q[10] = I * Pxy; q[11] = I * Pxs;
			q[12] = I * Pyy; q[13] = I * Pys;
			q[14] = I * Pss;
		};
		if (C.model == 6 || C.model == 7) {
			double sx = t[4], sy = t[4], dsx = 1, dsy = 1, ssx = 0, ssy = 0;
			if (C.model == 7) {
				AstigSigma(C.astig, C.pixelSize, t[4], sx, dsx, &ssx);
				AstigSigma(C.astig + 5, C.pixelSize, t[4], sy, dsy, &ssy);
			}
			std::vector<double> ex(roi), edx(roi), eds(roi), ey(roi), edy(roi), eys(roi), x2(3 * roi), y2(3 * roi);
			for (int j = 0; j < roi; ++j) { Erf1D(static_cast<double>(j - hh), t[2], sx, ex[j], edx[j], eds[j], h ? &x2[3 * j] : nullptr); }
			for (int i = 0; i < roi; ++i) { Erf1D(static_cast<double>(i - hh), t[3], sy, ey[i], edy[i], eys[i], h ? &y2[3 * i] : nullptr); }
			for (int i = 0; i < roi; ++i) {
				for (int j = 0; j < roi; ++j) {
					const int k = i * roi + j;
					const double psf = ex[j] * ey[i];
					mu[k] = t[0] + t[1] * psf;
					double* gk = g.data() + static_cast<size_t>(k) * 5;
					const double Px = edx[j] * ey[i], Py = ex[j] * edy[i];
					const double Ps = eds[j] * dsx * ey[i] + ex[j] * eys[i] * dsy;
					gk[0] = 1;
					gk[1] = psf;
					gk[2] = t[1] * Px;
					gk[3] = t[1] * Py;
					gk[4] = t[1] * Ps;
					if (h) {
						const double* X2 = &x2[3 * j];
						const double* Y2 = &y2[3 * i];
						const double Pxx = X2[0] * ey[i], Pxy = edx[j] * edy[i];
						const double Pxs = X2[1] * dsx * ey[i] + edx[j] * eys[i] * dsy;
						const double Pyy = ex[j] * Y2[0];
						const double Pys = eds[j] * dsx * edy[i] + ex[j] * Y2[1] * dsy;
						const double Pss = (X2[2] * dsx * dsx + eds[j] * ssx) * ey[i] + 2 * eds[j] * dsx * eys[i] * dsy +
						                   ex[j] * (Y2[2] * dsy * dsy + eys[i] * ssy);
						put2(k, Pxx, Pxy, Pxs, Pyy, Pys, Pss, Px, Py, Ps);
					}
				}
			}
			return;
		}
		const double X0 = (C.sx - 1) / 2.0, Y0 = (C.sy - 1) / 2.0;
		for (int i = 0; i < roi; ++i) {
			for (int j = 0; j < roi; ++j) {
				const int k = i * roi + j;
				double dX, dY, dZ, s2[6];
				const double psf = SplinePsf(C, X0 + (j - hh) - t[2], Y0 + (i - hh) - t[3], t[4], dX, dY, dZ, h ? s2 : nullptr);
				mu[k] = t[0] + t[1] * psf;
				double* gk = g.data() + static_cast<size_t>(k) * 5;
				gk[0] = 1;
				gk[1] = psf;
				gk[2] = -t[1] * dX;
				gk[3] = -t[1] * dY;
				gk[4] = t[1] * dZ;
				if (h) { put2(k, s2[0], s2[1], -s2[2], s2[3], -s2[4], s2[5], -dX, -dY, dZ); }
			}
		}
	}

	// Deviance D, gradient G and a 5x5 curvature matrix: Fisher scoring H = 2 sum dmu dmu^T / mu, or with `exact`
	// the Hessian of D, 2 sum [d / mu^2 dmu dmu^T + (1 - d / mu) d2mu].
	double Normal(const double* t, double G[5], double Hm[25], bool exact = false) const
	{
		std::vector<double> mu, g, h2;
		Eval(t, mu, g, exact ? &h2 : nullptr);
		double D = 0;
		for (int a = 0; a < 5; ++a) { G[a] = 0; }
		for (int a = 0; a < 25; ++a) { Hm[a] = 0; }
		for (int k = 0; k < c->n; ++k) {
			const double m = std::max(mu[k], 1e-6), dk = d[k];
			D += dk > 0 ? 2 * (m - dk - dk * std::log(m / dk)) : 2 * m;
			const double* gk = g.data() + static_cast<size_t>(k) * 5;
			const double w1 = 2 * (1 - dk / m), w2 = exact ? 2 * dk / (m * m) : 2 / m;
			int q = 0;
			for (int a = 0; a < 5; ++a) {
				G[a] += w1 * gk[a];
				for (int b = a; b < 5; ++b, ++q) {
					Hm[a * 5 + b] += w2 * gk[a] * gk[b];
					if (exact) { Hm[a * 5 + b] += w1 * h2[static_cast<size_t>(k) * 15 + q]; }
				}
			}
		}
		for (int a = 0; a < 5; ++a) {
			for (int b = 0; b < a; ++b) { Hm[a * 5 + b] = Hm[b * 5 + a]; }
		}
		return D;
	}
};

// Solves A x = b for a symmetric positive-definite 5x5 A; false if a pivot is not positive.
bool CholSolve5(const double* A, const double* b, double* x)
{
	double L[25] = {};
	for (int i = 0; i < 5; ++i) {
		for (int j = 0; j <= i; ++j) {
			double s = A[i * 5 + j];
			for (int k = 0; k < j; ++k) { s -= L[i * 5 + k] * L[j * 5 + k]; }
			if (i == j) {
				if (!(s > 0)) { return false; }
				L[i * 5 + i] = std::sqrt(s);
			}
			else { L[i * 5 + j] = s / L[j * 5 + j]; }
		}
	}
	double y[5];
	for (int i = 0; i < 5; ++i) {
		double s = b[i];
		for (int k = 0; k < i; ++k) { s -= L[i * 5 + k] * y[k]; }
		y[i] = s / L[i * 5 + i];
	}
	for (int i = 4; i >= 0; --i) {
		double s = y[i];
		for (int k = i + 1; k < 5; ++k) { s -= L[k * 5 + i] * x[k]; }
		x[i] = s / L[i * 5 + i];
	}
	return true;
}

void MleBounds(const MleCfg& c, double x0, double y0, double lo[5], double hi[5])
{
	const double h = static_cast<double>(c.half);
	lo[0] = 1e-3; hi[0] = 1e6;
	lo[1] = 1.0; hi[1] = 1e9;
	lo[2] = std::max(x0 - 2.0, -h); hi[2] = std::min(x0 + 2.0, h);
	lo[3] = std::max(y0 - 2.0, -h); hi[3] = std::min(y0 + 2.0, h);
	if (c.model == 6) { lo[4] = 0.5; hi[4] = 5.0; }
	else if (c.model == 7) { lo[4] = c.zMin; hi[4] = c.zMax; }
	else { lo[4] = 0.0; hi[4] = static_cast<double>(c.sz) - 1e-6; }
}

// Active bounds: a parameter that sits on a bound with the descent direction (-G) pointing outside is held there -
// its row and column of the system become those of the identity and its right-hand side zero - so that the step of
// the other parameters is the minimiser of the model restricted to them instead of a clipped full step.
void FixActive(const double* t, const double* G, const double* lo, const double* hi, double* A, double* rhs)
{
	for (int a = 0; a < 5; ++a) {
		if ((t[a] <= lo[a] && G[a] > 0) || (t[a] >= hi[a] && G[a] < 0)) {
			for (int b = 0; b < 5; ++b) { A[a * 5 + b] = 0; A[b * 5 + a] = 0; }
			A[a * 5 + a] = 1;
			rhs[a] = 0;
		}
	}
}

// LM stop rule: an accepted step below 1e-4 px in x and y, 1e-4 relative in I, bg (floor 1) and the width / z
// coordinate (1e-4 px for sigma, 1e-2 nm for z in nm, 1e-4 table units for the spline z).
bool MleStepSmall(const MleCfg& c, const double* a, const double* b)
{
	const double sTol = c.model == 7 ? 1e-2 : 1e-4;
	return std::abs(b[2] - a[2]) < 1e-4 && std::abs(b[3] - a[3]) < 1e-4 && std::abs(b[1] - a[1]) < 1e-4 * std::max(std::abs(a[1]), 1.0) &&
	       std::abs(b[0] - a[0]) < 1e-4 * std::max(std::abs(a[0]), 1.0) && std::abs(b[4] - a[4]) < sTol;
}

// The fit of one candidate (coordinates local to the integer ROI centre); returns false for a failed fit.
bool MleFit(const MleRoi& R, double t[5], double crlb[5], double& dev)
{
	const MleCfg& c = *R.c;
	double lo[5], hi[5];
	MleBounds(c, R.x0, R.y0, lo, hi);
	double dmin = 1e300, sum = 0;
	for (double v : R.d) { dmin = std::min(dmin, v); sum += v; }
	t[0] = std::max(dmin, 1e-3);
	t[1] = std::max(sum - t[0] * c.n, 1.0);
	t[2] = R.x0;
	t[3] = R.y0;
	if (c.model == 6) { t[4] = c.sigma0; }
	else {
		// coarse scan of the axial parameter at the initial bg, I, x, y (16 points for mode 7, 8 for mode 8)
		const int ns = c.model == 7 ? 16 : 8;
		double best = 1e300, bz = 0.5 * (lo[4] + hi[4]);
		for (int k = 0; k < ns; ++k) {
			t[4] = lo[4] + (hi[4] - lo[4]) * (k + 0.5) / ns;
			double G[5], Hm[25];
			const double D = R.Normal(t, G, Hm);
			if (D < best) { best = D; bz = t[4]; }
		}
		t[4] = bz;
	}
	for (int a = 0; a < 5; ++a) { t[a] = std::min(std::max(t[a], lo[a]), hi[a]); }
	double G[5], Hm[25];
	double D = R.Normal(t, G, Hm);
	if (!std::isfinite(D)) { return false; }
	double lambda = 1e-3;
	for (int it = 0; it < c.maxIter; ++it) {
		double A[25], rhs[5], dt[5];
		for (int a = 0; a < 25; ++a) { A[a] = Hm[a]; }
		for (int a = 0; a < 5; ++a) { A[a * 5 + a] *= 1.0 + lambda; rhs[a] = -G[a]; }
		FixActive(t, G, lo, hi, A, rhs);
		if (!CholSolve5(A, rhs, dt)) {
			lambda *= 10;
			if (lambda > 1e7) { break; }
			continue;
		}
		double tt[5];
		for (int a = 0; a < 5; ++a) { tt[a] = std::min(std::max(t[a] + dt[a], lo[a]), hi[a]); }
		double Gt[5], Ht[25];
		const double Dt = R.Normal(tt, Gt, Ht);
		if (std::isfinite(Dt) && Dt < D) {
			const bool small = MleStepSmall(c, t, tt);
			for (int a = 0; a < 5; ++a) { t[a] = tt[a]; G[a] = Gt[a]; }
			for (int a = 0; a < 25; ++a) { Hm[a] = Ht[a]; }
			D = Dt;
			lambda = std::max(lambda * 0.1, 1e-7);
			if (small) { break; }
		}
		else {
			lambda *= 10;
			if (lambda > 1e7) { break; }
		}
	}
	// Newton steps on the exact Hessian of the deviance in FP64 (Fisher scoring where that Hessian is not positive
	// definite) until the relative step is below 1e-10, at most 6 steps; a step that does not lower the deviance is
	// halved up to three times
	D = R.Normal(t, G, Hm, true);
	for (int it = 0; it < 6; ++it) {
		double rhs[5], dt[5], tt[5], A[25];
		for (int a = 0; a < 5; ++a) { rhs[a] = -G[a]; }
		for (int a = 0; a < 25; ++a) { A[a] = Hm[a]; }
		FixActive(t, G, lo, hi, A, rhs);
		if (!CholSolve5(A, rhs, dt)) {
			double Gf[5], Hf[25];
			R.Normal(t, Gf, Hf, false);
			FixActive(t, G, lo, hi, Hf, rhs);
			if (!CholSolve5(Hf, rhs, dt)) { break; }
		}
		bool accepted = false;
		double Gt[5], Ht[25], Dt = 0;
		for (int half = 0; half < 4 && !accepted; ++half) {
			for (int a = 0; a < 5; ++a) { tt[a] = std::min(std::max(t[a] + dt[a], lo[a]), hi[a]); }
			Dt = R.Normal(tt, Gt, Ht, true);
			if (std::isfinite(Dt) && Dt <= D) { accepted = true; }
			else { for (int a = 0; a < 5; ++a) { dt[a] *= 0.5; } }
		}
		if (!accepted) { break; }
		double step = 0;
		for (int a = 0; a < 5; ++a) { step = std::max(step, std::abs(tt[a] - t[a]) / std::max(std::abs(t[a]), 1.0)); }
		for (int a = 0; a < 5; ++a) { t[a] = tt[a]; G[a] = Gt[a]; }
		for (int a = 0; a < 25; ++a) { Hm[a] = Ht[a]; }
		D = Dt;
		if (step < 1e-10) { break; }
	}
	R.Normal(t, G, Hm, false);  // Fisher information for the CRLB
	// CRLB: Fisher information F = H / 2; variances are the diagonal of its inverse
	for (int a = 0; a < 5; ++a) {
		double e[5] = {0, 0, 0, 0, 0}, col[5], F[25];
		for (int q = 0; q < 25; ++q) { F[q] = 0.5 * Hm[q]; }
		e[a] = 1;
		if (!CholSolve5(F, e, col)) { return false; }
		crlb[a] = col[a] > 0 ? std::sqrt(col[a]) : 0.0;
	}
	dev = D;
	for (int a = 0; a < 5; ++a) { if (!std::isfinite(t[a])) { return false; } }
	return true;
}

// ROI photons and local candidate position; false when the ROI crosses the frame border (Fitting.cpp's test).
bool MleRoiAt(const MleCfg& c, const uint16_t* img, int W, int H, double cx, double cy, MleRoi& R)
{
	const size_t ux = static_cast<size_t>(cx), uy = static_cast<size_t>(cy);
	const size_t h = static_cast<size_t>(c.half);
	const bool nonneg = cx >= 0 && cy >= 0;
	if (!nonneg || h > ux || ux >= static_cast<size_t>(W) - h || h > uy || uy >= static_cast<size_t>(H) - h) { return false; }
	R.c = &c;
	R.d.resize(c.n);
	for (int i = 0; i < c.roi; ++i) {
		for (int j = 0; j < c.roi; ++j) {
			const double adu = static_cast<double>(img[(uy - h + i) * static_cast<size_t>(W) + (ux - h + j)]);
			R.d[i * c.roi + j] = std::max((adu - c.offset) / c.gain, 0.0);
		}
	}
	R.x0 = cx - static_cast<double>(ux);
	R.y0 = cy - static_cast<double>(uy);
	return true;
}

void FitMle(const MleCfg& c, const uint16_t* img, int W, int H, const Candidate& cd, Row& out)
{
	const size_t ux = static_cast<size_t>(cd.x), uy = static_cast<size_t>(cd.y);
	MleRoi R;
	if (!MleRoiAt(c, img, W, H, cd.x, cd.y, R)) {
		FillRow(kG2Sigma, cd, out, cd.x, cd.y, 0);
		return;
	}
	double t[5], crlb[5], dev = 0;
	const bool ok = MleFit(R, t, crlb, dev);
	const double qxy = std::sqrt(0.5 * (crlb[2] * crlb[2] + crlb[3] * crlb[3]));
	if (!ok || (c.crlbMax > 0 && !(qxy <= c.crlbMax))) {
		FillRow(kG2Sigma, cd, out, cd.x, cd.y, 0);
		return;
	}
	double sx = t[4], sy = t[4], z = 0, qz = -1;
	if (c.model == 7) {
		double d1, d2;
		AstigSigma(c.astig, c.pixelSize, t[4], sx, d1);
		AstigSigma(c.astig + 5, c.pixelSize, t[4], sy, d2);
		z = t[4];
		qz = crlb[4];
	}
	if (c.model == 8) { sx = sy = 0; z = c.dz * (t[4] - c.sz / 2.0); qz = c.dz * crlb[4]; }
	out[cId] = 0; out[cPlane] = 0; out[cIndex] = 0; out[cChannel] = -1;
	out[cX] = static_cast<double>(ux) + t[2];
	out[cY] = static_cast<double>(uy) + t[3];
	out[cZ] = z;
	out[cIntensity] = t[1];
	// Theta (no rotation in these models): the FP64 deviance at the result, the fit's log-likelihood ratio
	out[cSigmaX] = sx; out[cSigmaY] = sy; out[cTheta] = dev;
	out[cQualityXY] = qxy; out[cQualityZ] = qz;
	out[cAmplitude] = (sx > 0 && sy > 0) ? t[1] / (6.283185307179586 * sx * sy) : t[1];
	out[cOffset] = t[0];
	out[cSegIntensity] = cd.intensity; out[cSurface] = cd.surf;
	out[cCircularity] = (sx > kEps && sy > kEps) ? std::min(sx, sy) / std::max(sx, sy) : 1;
}

}  // namespace

namespace {

// Strict weak order on (Y, X) with std::weak_order semantics (FrameProcessor.cpp:35-39).
bool RowLess(const Row& a, const Row& b)
{
	if (const auto o = std::weak_order(a[cY], b[cY]); o != 0) { return o < 0; }
	return std::weak_order(a[cX], b[cX]) < 0;
}

// One frame: wavelet -> segmentation -> fits of the first maxPoints candidates -> sort (FrameProcessor.cpp:28-82).
void ProcessFrame(const uint16_t* img, int H, int W, double thr, double ratio, size_t maxPoints, int fit, const double* fp,
                  std::vector<Row>& rows)
{
	std::vector<double> planes[kNumPlanes];
	Atrous(img, H, W, planes);
	Segmenter seg;
	seg.Run(planes[kPlaneId].data(), H, W, thr, ratio);
	const size_t count = std::min(seg.cands.size(), maxPoints);
	if (seg.cands.size() > maxPoints) { std::fprintf(stderr, "[WARNING] Density is too high; some points are missed (output capacity exceeded).\n"); }
	rows.assign(count, Row{});
	const int mode = (fit >= 1 && fit <= 8) ? fit : kNone;
	if (mode >= 6) {
		MleCfg mc;
		ParseMle(mode, fp, mc);
		for (size_t i = 0; i < count; ++i) { FitMle(mc, img, W, H, seg.cands[i], rows[i]); }
	}
	else if (mode >= kG2Fixed && mode <= kG3Theta) {
		FitConfig cf;
		cf.Init(mode, fp, img, W, H);
		for (size_t i = 0; i < count; ++i) { FitGaussian(cf, seg.cands[i], rows[i]); }
	}
	else if (mode == kSplineEmccd) {
		SplineTable t;
		t.Init(fp);
		for (size_t i = 0; i < count; ++i) { FitSplineFull(t, fp[0], img, W, H, seg.cands[i], rows[i]); }
	}
	else {
		for (size_t i = 0; i < count; ++i) {
			const Candidate& c = seg.cands[i];
			FillRow(kNone, c, rows[i], c.x, c.y, c.z, 0, 0);
		}
	}
	std::sort(rows.begin(), rows.end(), RowLess);
}

}  // namespace

namespace {

// ---------------------------------------------------------------------------------------------
// Spline calibration: the cubic B-spline coefficient table of a PSF volume (lib/signal_processing/BSpline3D.cpp,
// constructed by the calibration at lib/signal_processing/Spline.cpp:52 with degree 3 and lambda = {0, 0, 100 / dz}).
// Degree 3 only (the degree the calibration uses). Steps of BSpline3D::BSpline3D (:17-45):
//   1. per axis, the exponential filters of its poles (getPolesFilter :171-214: lambda = 0 -> pole sqrt3 - 2, gain 6;
//      lambda > 0 -> the roots of 1 - 4z + 6z^2 - 4z^3 + z^4 + (z + 4z^2 + z^3) / (6 lambda) with |z| <= 1 from
//      Durand-Kerner (solvePolynomial :372-430), gain 1 / lambda), applied along every line with mirror
//      initialisation over K0 = ceil(log(eps) / log|z|) terms (applyFilter :284-331, symExpFilt :438-449; Unser,
//      Aldroubi & Eden 1991), the real part times the gain kept after each axis;
//   2. reflection padding by one voxel (:23-41, Matrix.cpp ReflectIndex1D :426-444);
//   3. the spline's values at the voxel centres (interpolateHDR :334-348, interpolate_at :351-385);
//   4. those values upsampled by 3 as cubic B-spline control points with zeros outside
//      (Interpolation3D::Upsample :188-229 with spline3D :114-145), and per cell the 64 monomial coefficients that
//      reproduce its 4 x 4 x 4 samples, A^-1 samples with the Gauss-Jordan inverse of A (getFinalCoeff :99-164).
// Coefficient k = l * 16 + m * 4 + n of cell (x, y, z) multiplies zf^l yf^m xf^n (the reference's naming: its "Dx"
// runs along z).

// BSpline3D::Eval(x, 3) (BSpline3D.cpp:76-88), same operations and order.
double Bspline3(double x)
{
	constexpr double Edge = 4.0 / 3.0, Center = 2.0 / 3.0, A = 2.0, C = 1.0 / 6.0, D = 0.5;
	const double X2 = x * x, X3 = X2 * x;
	if (x >= -2 && x < -1) { return Edge + (A * x) + X2 + (C * X3); }
	if (x >= -1 && x < 0) { return Center - X2 - (D * X3); }
	if (x >= 0 && x < 1) { return Center - X2 + (D * X3); }
	if (x >= 1 && x < 2) { return Edge - (A * x) + X2 - (C * X3); }
	return 0;
}

using cplx = std::complex<double>;

// Durand-Kerner roots of a real polynomial (coefficients from the highest degree), as solvePolynomial does for
// degrees other than 3: 0.4 e^{2 pi i k / deg} start, simultaneous updates, stop when every |delta| <= tol.
std::vector<cplx> DurandKerner(const std::vector<double>& c, double tol = 1e-12, int maxIter = 100)
{
	const size_t deg = c.size() - 1;
	std::vector<cplx> roots(deg);
	for (size_t k = 0; k < deg; ++k) {
		const double th = 2.0 * std::numbers::pi * static_cast<double>(k) / static_cast<double>(deg);
		roots[k] = 0.4 * cplx(std::cos(th), std::sin(th));
	}
	auto eval = [&](cplx x) {
		cplx v = 0.0;
		for (size_t i = 0; i <= deg; ++i) { v += c[i] * std::pow(x, static_cast<int>(deg - i)); }
		return v;
	};
	for (int it = 0; it < maxIter; ++it) {
		bool converged = true;
		std::vector<cplx> next = roots;
		for (size_t i = 0; i < deg; ++i) {
			cplx den = 1.0;
			for (size_t j = 0; j < deg; ++j) {
				if (j != i) { den *= roots[i] - roots[j]; }
			}
			const cplx d = eval(roots[i]) / den;
			next[i] = roots[i] - d;
			if (std::abs(d) > tol) { converged = false; }
		}
		roots = next;
		if (converged) { break; }
	}
	return roots;
}

// Poles and gain of the degree-3 smoothing-spline filter for one axis (getPolesFilter, case 3).
void CubicPoles(double lambda, std::vector<cplx>& poles, double& gain)
{
	poles.clear();
	if (lambda <= std::numeric_limits<double>::epsilon()) {
		poles.emplace_back(std::numbers::sqrt3 - 2.0);
		gain = 6.0;
		return;
	}
	std::vector<double> p{1, -4, 6, -4, 1};
	p[1] += 1.0 / (6.0 * lambda);
	p[2] += 2.0 / (3.0 * lambda);
	p[3] += 1.0 / (6.0 * lambda);
	for (const cplx& z : DurandKerner(p)) {
		if (std::abs(z) <= 1.0) { poles.push_back(z); }
	}
	gain = 1.0 / lambda;
}

// Mirror index sequence 0, 1, .., n-1, n-2, .., 1, 0, 1, .. (Matrix.cpp ReflectionIndices :413-423), entry k.
size_t Reflection(size_t n, size_t k) { return n == 1 ? 0 : (k % (2 * n - 2) < n ? k % (2 * n - 2) : 2 * n - 2 - k % (2 * n - 2)); }

// One line through the symmetric exponential filter of pole z (symExpFilt).
void SymExpFilt(std::vector<cplx>& x, cplx z, size_t k0)
{
	const size_t n = x.size();
	const cplx c0 = -z / (1.0 - z * z);
	std::vector<cplx> y(n, 0.0);
	for (size_t k = 0; k < k0; ++k) { y[0] += std::pow(z, static_cast<int>(k)) * x[Reflection(n, k)]; }
	for (size_t k = 1; k < n; ++k) { y[k] = x[k] + z * y[k - 1]; }
	y[n - 1] = (2.0 * y[n - 1] - x[n - 1]) * c0;
	for (int k = static_cast<int>(n) - 2; k >= 0; --k) { y[k] = (y[k + 1] - y[k]) * z; }
	x.swap(y);
}

// coeffs [nz][ny][nx] filtered along `axis` (0 x, 1 y, 2 z) by every pole, then real part times the gain (applyFilter).
void FilterAxis(std::vector<double>& coeffs, const size_t dim[3], int axis, const std::vector<cplx>& poles, double gain)
{
	const size_t nx = dim[0], ny = dim[1], nz = dim[2];
	const size_t n = dim[axis];
	std::vector<cplx> tmp(coeffs.begin(), coeffs.end()), line(n);
	auto at = [&](size_t x, size_t y, size_t z) { return (z * ny + y) * nx + x; };
	const double k0tol = std::log(std::numeric_limits<double>::epsilon());
	for (const cplx& z : poles) {
		const auto k0 = static_cast<size_t>(std::ceil(k0tol / std::log(std::abs(z))));
		const size_t outerA = axis == 2 ? ny : nz, outerB = axis == 0 ? ny : nx;
		for (size_t a = 0; a < outerA; ++a) {
			for (size_t b = 0; b < outerB; ++b) {
				auto idx = [&](size_t i) {
					return axis == 0 ? at(i, b, a) : axis == 1 ? at(b, i, a) : at(b, a, i);
				};
				for (size_t i = 0; i < n; ++i) { line[i] = tmp[idx(i)]; }
				SymExpFilt(line, z, k0);
				for (size_t i = 0; i < n; ++i) { tmp[idx(i)] = line[i]; }
			}
		}
	}
	for (size_t i = 0; i < coeffs.size(); ++i) { coeffs[i] = std::real(tmp[i]) * gain; }
}

}  // namespace

extern "C" {

void orc_SetThreads(int n) { if (n > 0) { omp_set_num_threads(n); } }

// Localization (CPU/main.cpp:112-121 -> lib/Palm.cpp:48-70, 24-43).
uint64_t orc_Localization(const uint16_t* input, double* output, uint64_t outputSize, uint64_t height, uint64_t width,
                          uint64_t planes, double thr, double ratio, uint64_t fit, const double* fp)
{
	const size_t perPlane = planes == 0 ? 0 : (outputSize / kCols) / planes;
	if (perPlane == 0) { return 0; }
	const size_t frame = static_cast<size_t>(height) * width;
	std::vector<std::vector<Row>> all(planes);
	#pragma omp parallel for schedule(dynamic, 1)
	for (int64_t z = 0; z < static_cast<int64_t>(planes); ++z) {
		ProcessFrame(input + z * frame, static_cast<int>(height), static_cast<int>(width), thr, ratio, perPlane,
		             static_cast<int>(fit), fp, all[z]);
	}
	size_t count = 0, id = 1;
	for (size_t z = 0; z < planes; ++z) {
		size_t local = 1;
		for (const Row& r : all[z]) {
			std::copy(r.begin(), r.end(), output + count);
			output[count + cId] = static_cast<double>(id++);
			output[count + cPlane] = static_cast<double>(z + 1);
			output[count + cIndex] = static_cast<double>(local++);
			count += kCols;
		}
	}
	return count;
}

// Fit-only at given positions (CPU/main.cpp:141-148 -> lib/Palm.cpp:73-119). Fit 0 is not supported by the
// reference here (its GaussianFit throws for the "none" model); this restatement fills no-fit rows for it.
uint64_t orc_Fitting(const uint16_t* input, const double* positions, uint64_t nPoints, double* output, uint64_t /*outputSize*/,
                     uint64_t height, uint64_t width, uint64_t planes, uint64_t fit, const double* fp)
{
	if (nPoints == 0) { return 0; }
	std::vector<size_t> localIdx(nPoints), perPlane(planes, 0);
	for (size_t i = 0; i < nPoints; ++i) { localIdx[i] = ++perPlane[static_cast<size_t>(positions[i * 6 + 1]) - 1]; }
	const size_t frame = static_cast<size_t>(height) * width;
	#pragma omp parallel for schedule(static)
	for (int64_t i = 0; i < static_cast<int64_t>(nPoints); ++i) {
		const double* pos = positions + i * 6;
		const size_t plane = static_cast<size_t>(pos[1]) - 1;
		const uint16_t* img = input + plane * frame;
		Candidate c;
		c.x = pos[2]; c.y = pos[3]; c.intensity = pos[4]; c.surf = pos[5];
		Row r{};
		if (fit >= 6 && fit <= 8) {
			MleCfg mc;
			ParseMle(static_cast<int>(fit), fp, mc);
			FitMle(mc, img, static_cast<int>(width), static_cast<int>(height), c, r);
		}
		else if (fit == kSplineEmccd) {
			SplineTable t;
			t.Init(fp);
			FitSplineFull(t, fp[0], img, static_cast<int>(width), static_cast<int>(height), c, r);
		}
		else if (fit >= 1 && fit <= 4) {
			FitConfig cf;
			cf.Init(static_cast<int>(fit), fp, img, static_cast<int>(width), static_cast<int>(height));
			FitGaussian(cf, c, r);
		}
		else { FillRow(kNone, c, r, c.x, c.y, c.z, 0, 0); }
		r[cId] = pos[0];
		r[cPlane] = pos[1];
		r[cIndex] = static_cast<double>(localIdx[i]);
		std::copy(r.begin(), r.end(), output + i * kCols);
	}
	return nPoints * kCols;
}

// Wavelett (CPU/main.cpp:257-284).
void orc_Wavelett(const uint16_t* input, double* output, uint64_t height, uint64_t width, uint64_t planes, uint64_t level)
{
	if (planes == 0) { return; }
	if (level == 0) { level = 1; }
	const uint64_t lv = std::min<uint64_t>(level - 1, kNumPlanes - 1);
	const size_t frame = static_cast<size_t>(height) * width;
	#pragma omp parallel for schedule(static)
	for (int64_t z = 0; z < static_cast<int64_t>(planes); ++z) {
		std::vector<double> pl[kNumPlanes];
		Atrous(input + z * frame, static_cast<int>(height), static_cast<int>(width), pl);
		std::copy(pl[lv].begin(), pl[lv].end(), output + z * frame);
	}
}

// AutoThreshold on frame 0 (CPU/main.cpp:75-85 -> lib/Palm.cpp:122-172).
double orc_AutoThreshold(const uint16_t* input, uint64_t height, uint64_t width, const double* fp)
{
	const size_t size = static_cast<size_t>(height) * width;
	const auto cap = static_cast<uint64_t>(0.2 * static_cast<double>(height * width) * kCols);
	const size_t maxPoints = cap / kCols;
	const double halfRoi = fp[0] / 2;
	double mu = 0.0;
	for (size_t i = 0; i < size; ++i) { mu += input[i]; }
	mu /= static_cast<double>(size);
	double var = 0.0;
	for (size_t i = 0; i < size; ++i) { var += (input[i] - mu) * (input[i] - mu); }
	var /= static_cast<double>(size);
	double thr = std::sqrt(var);
	std::vector<char> mask(size);
	std::vector<Row> pts;
	const int W = static_cast<int>(width), H = static_cast<int>(height);
	for (int iter = 0; iter < kThresholdIters; ++iter) {
		ProcessFrame(input, H, W, thr, 10, maxPoints, 0, fp, pts);
		std::fill(mask.begin(), mask.end(), 0);
		for (const Row& p : pts) {
			const auto x0 = static_cast<size_t>(std::max(0, static_cast<int>(p[cX] - halfRoi)));
			const auto x1 = std::min(static_cast<size_t>(W), static_cast<size_t>(p[cX] + halfRoi));
			const auto y0 = static_cast<size_t>(std::max(0, static_cast<int>(p[cY] - halfRoi)));
			const auto y1 = std::min(static_cast<size_t>(H), static_cast<size_t>(p[cY] + halfRoi));
			for (size_t yy = y0; yy < y1; ++yy) { for (size_t xx = x0; xx < x1; ++xx) { mask[yy * width + xx] = 1; } }
		}
		size_t count = 0;
		double sum = 0;
		for (size_t j = 0; j < size; ++j) { if (!mask[j]) { sum += input[j]; ++count; } }
		if (count == 0) { break; }
		mu = sum / static_cast<double>(count);
		var = 0.0;
		for (size_t j = 0; j < size; ++j) { if (!mask[j]) { var += (input[j] - mu) * (input[j] - mu); } }
		var /= static_cast<double>(count);
		var = std::sqrt(var);
		if (std::abs(thr - var) <= std::numeric_limits<double>::epsilon()) { break; }
		thr = var;
	}
	return thr;
}

// All wavelet planes of one frame (planes[k*H*W + p]).
void orc_Planes(const uint16_t* frame, uint64_t height, uint64_t width, double* out)
{
	std::vector<double> pl[kNumPlanes];
	Atrous(frame, static_cast<int>(height), static_cast<int>(width), pl);
	const size_t n = static_cast<size_t>(height) * width;
	for (int k = 0; k < kNumPlanes; ++k) { std::copy(pl[k].begin(), pl[k].end(), out + k * n); }
}

static uint64_t DumpCandidates(const Segmenter& seg, double* rows, uint64_t capacity)
{
	for (size_t i = 0; i < seg.cands.size() && i < capacity; ++i) {
		rows[4 * i + 0] = seg.cands[i].x;
		rows[4 * i + 1] = seg.cands[i].y;
		rows[4 * i + 2] = seg.cands[i].intensity;
		rows[4 * i + 3] = seg.cands[i].surf;
	}
	return seg.cands.size();
}

// Segmentation candidates of one frame in label order: rows (x, y, intensity, surf).
uint64_t orc_Candidates(const uint16_t* frame, uint64_t height, uint64_t width, double thr, double ratio, double* rows,
                        uint64_t capacity)
{
	std::vector<double> pl[kNumPlanes];
	Atrous(frame, static_cast<int>(height), static_cast<int>(width), pl);
	Segmenter seg;
	seg.Run(pl[kPlaneId].data(), static_cast<int>(height), static_cast<int>(width), thr, ratio);
	return DumpCandidates(seg, rows, capacity);
}

uint64_t orc_CandidatesFromPotential(const double* potential, uint64_t height, uint64_t width, double thr, double ratio,
                                     double* rows, uint64_t capacity)
{
	Segmenter seg;
	seg.Run(potential, static_cast<int>(height), static_cast<int>(width), thr, ratio);
	return DumpCandidates(seg, rows, capacity);
}

// Final label map of one frame after the watershed stages, before the surface filter (labels 1..n, 0 = none).
uint64_t orc_Labels(const uint16_t* frame, uint64_t height, uint64_t width, double thr, double ratio, uint32_t* labels)
{
	std::vector<double> pl[kNumPlanes];
	Atrous(frame, static_cast<int>(height), static_cast<int>(width), pl);
	Segmenter seg;
	seg.H = static_cast<int>(height);
	seg.W = static_cast<int>(width);
	seg.ratio = ratio;
	const size_t n = static_cast<size_t>(height) * width;
	seg.pot.assign(n, 0.0);
	seg.lab.assign(n, 0);
	for (size_t i = 0; i < n; ++i) { seg.pot[i] = pl[kPlaneId][i] > thr ? pl[kPlaneId][i] : 0.0; }
	seg.Seeds();
	seg.Flood();
	if (static_cast<int>(ratio) > 0) { seg.Fuse(); seg.Flood(); }
	std::copy(seg.lab.begin(), seg.lab.end(), labels);
	return seg.cands.size();
}

// z from the fitted widths (AstigFit::Estimate, lib/fit/AstigFit.cpp:36-59, exported as Astigmatism3DEstimation,
// CPU/main.cpp:324-353). Per point: the squared width error over a 201-point grid of [-zMax, zMax], Brent's
// minimisation (golden section with parabolic steps, Brent 1973) on the best grid point +-2 grid steps (:342-447,
// constants AstigFit.hpp:110-114), the grid point kept when Brent does not improve on it, and the compatibility
// score 1 / (1 + (Rx^2 + Ry^2) / 2), R = relative width error / 0.2 (:99-109). Widths from the model
// sigma_px = A / pixelSize * sqrt(max(0, 1 + U^2 + c3 U^3 + c4 U^4)), U = (z - z0) / w (:76-88).
// input [size][2] = (sigma_x, sigma_y) px, output [size][2] = (z nm, score), model [z0, w, c3, c4, A] x then y.
void orc_Astig3DEstimation(const double* input, double* output, uint64_t size, double pixelSize, const double* model, double zMax)
{
	struct Axis { double z0, w, c3, c4, a; };
	const Axis ax[2] = {{model[0], model[1], model[2], model[3], model[4]}, {model[5], model[6], model[7], model[8], model[9]}};
	const double scale = 1.0 / pixelSize;  // sampling (1) over the pixel size, then times the width in nm
	auto width = [&](const Axis& m, double z) {
		const double u = (z - m.z0) / m.w;
		const double u2 = u * u, u3 = u2 * u, u4 = u3 * u;
		const double poly = 1.0 + u2 + (m.c3 * u3) + (m.c4 * u4);
		return scale * (m.a * std::sqrt(std::max(0.0, poly)));
	};
	auto err = [&](double z, double sx, double sy) {
		const double dx = width(ax[0], z) - sx, dy = width(ax[1], z) - sy;
		return (dx * dx) + (dy * dy);
	};
	constexpr int kGrid = 201, kIter = 80;
	constexpr double kTol = 1e-3, kZTol = 1e-9, kQ = 0.2;
	const double lo = -zMax, hi = zMax, span = hi - lo;
	#pragma omp parallel for
	for (long long i = 0; i < static_cast<long long>(size); ++i) {
		const double sx = input[2 * i], sy = input[2 * i + 1];
		double bestZ = lo, bestE = std::numeric_limits<double>::infinity();
		for (int g = 0; g < kGrid; ++g) {
			const double z = lo + ((static_cast<double>(g) / static_cast<double>(kGrid - 1)) * span);
			const double e = err(z, sx, sy);
			if (e < bestE) { bestE = e; bestZ = z; }
		}
		const double step = span / static_cast<double>(kGrid - 1);
		double a = std::max(lo, std::min(bestZ - (2.0 * step), hi));
		double b = std::max(lo, std::min(bestZ + (2.0 * step), hi));
		if (b < a) { std::swap(a, b); }
		// Brent: x best point so far, w second best, v the previous w; d the last step, e the one before
		constexpr double kGold = 1.0 - 0.6180339887498948482;
		double x = a + (kGold * (b - a)), w = x, v = x;
		double fx = err(x, sx, sy), fw = fx, fv = fx, d = 0.0, e = 0.0;
		double rz = x, rf = fx;
		bool stopped = false;
		for (int it = 0; it < kIter && !stopped; ++it) {
			const double mid = 0.5 * (a + b);
			const double tol1 = (kTol * std::abs(x)) + 1e-12, tol2 = 2.0 * tol1;
			if (std::abs(x - mid) <= tol2 - (0.5 * (b - a))) { stopped = true; break; }
			bool para = false;
			if (std::abs(e) > tol1) {
				const double r = (x - w) * (fx - fv);
				double q = (x - v) * (fx - fw);
				double p = ((x - v) * q) - ((x - w) * r);
				q = 2.0 * (q - r);
				if (q > 0.0) { p = -p; }
				q = std::abs(q);
				const double eOld = e;
				e = d;
				if (std::abs(p) < std::abs(0.5 * q * eOld) && p > q * (a - x) && p < q * (b - x)) {
					para = true;
					d = p / q;
					const double u = x + d;
					if (u - a < tol2 || b - u < tol2) { d = x < mid ? tol1 : -tol1; }
				}
			}
			if (!para) {
				e = x < mid ? b - x : a - x;
				d = kGold * e;
			}
			const double u = x + (std::abs(d) >= tol1 ? d : (d > 0.0 ? tol1 : -tol1));
			const double fu = err(u, sx, sy);
			if (fu <= fx) {
				if (u < x) { b = x; } else { a = x; }
				v = w; fv = fw; w = x; fw = fx; x = u; fx = fu;
			}
			else {
				if (u < x) { a = u; } else { b = u; }
				if (fu <= fw || std::abs(x - w) <= kZTol) { v = w; fv = fw; w = u; fw = fu; }
				else if (fu <= fv || std::abs(v - x) <= kZTol || std::abs(v - w) <= kZTol) { v = u; fv = fu; }
			}
		}
		rz = x;
		rf = fx;
		const double z = rf < bestE ? rz : bestZ;
		const double px = width(ax[0], z), py = width(ax[1], z);
		double score = 0.0;
		if (std::isfinite(px) && std::isfinite(py) && px > 0 && py > 0 && std::isfinite(sx) && std::isfinite(sy) && sx > 0 && sy > 0) {
			const double rx = (sx - px) / px / kQ, ry = (sy - py) / py / kQ;
			score = 1.0 / (1.0 + (0.5 * ((rx * rx) + (ry * ry))));
		}
		output[2 * i] = z;
		output[2 * i + 1] = score;
	}
}

// Analysis helpers for the maximum-likelihood modes 6-8 (fit_params as for orc_Localization); theta is local to
// the integer ROI centre floor(cx), floor(cy). Both return 0 when the ROI crosses the frame border.
// orc_MleEvaluate: FP64 deviance, gradient and exact Hessian (row-major 5x5) at theta.
int orc_MleEvaluate(const uint16_t* frame, uint64_t height, uint64_t width, double cx, double cy, uint64_t fit, const double* fp,
                    const double* theta, double* D, double* G, double* Hm)
{
	MleCfg c;
	if (fit < 6 || fit > 8 || !ParseMle(static_cast<int>(fit), fp, c)) { return 0; }
	MleRoi R;
	if (!MleRoiAt(c, frame, static_cast<int>(width), static_cast<int>(height), cx, cy, R)) { return 0; }
	*D = R.Normal(theta, G, Hm, true);
	return 1;
}

// orc_MleFitOne: the fit of one candidate (theta, CRLB, final deviance); returns 1 for a successful fit, 2 for a
// failed one.
int orc_MleFitOne(const uint16_t* frame, uint64_t height, uint64_t width, double cx, double cy, uint64_t fit, const double* fp,
                  double* theta, double* crlb, double* dev)
{
	MleCfg c;
	if (fit < 6 || fit > 8 || !ParseMle(static_cast<int>(fit), fp, c)) { return 0; }
	MleRoi R;
	if (!MleRoiAt(c, frame, static_cast<int>(width), static_cast<int>(height), cx, cy, R)) { return 0; }
	return MleFit(R, theta, crlb, *dev) ? 1 : 2;
}

// Frame-to-frame linking (Tracks::Tracking, lib/tracking/Tracks.cpp:69-212, exported as Tracking, CPU/main.cpp:159-164).
// Points (Id, Plane, X, Y) ordered by (Plane, Id) (:80-98; equal pairs by input position here, unspecified there);
// for every two consecutive planes that both hold points, the pairs with (xa - xb)^2 + (ya - yb)^2 <= maxDistance^2
// (:131-145) in increasing (d2, source, target) order link when the source has no successor and the target no
// predecessor yet (:148-186); track numbers 1, 2, ... go to the chain heads in point order and along their chains
// (:188-199). output [n][2] = (Id, Track) in point order; returns 2 n.
uint64_t orc_Tracking(const double* input, uint64_t* output, uint64_t nPoints, double maxDistance)
{
	if (nPoints == 0) { return 0; }
	struct Pt {
		size_t plane, id, src;
		double x, y;
	};
	std::vector<Pt> pts(nPoints);
	for (size_t i = 0; i < nPoints; ++i) {
		const double* r = input + 4 * i;
		pts[i] = {static_cast<size_t>(r[1]), static_cast<size_t>(r[0]), i, r[2], r[3]};
	}
	std::sort(pts.begin(), pts.end(), [](const Pt& a, const Pt& b) {
		if (a.plane != b.plane) { return a.plane < b.plane; }
		if (a.id != b.id) { return a.id < b.id; }
		return a.src < b.src;
	});
	constexpr size_t kNone = std::numeric_limits<size_t>::max();
	std::vector<size_t> succ(nPoints, kNone), pred(nPoints, kNone), track(nPoints, 0);
	const double r2 = maxDistance * maxDistance;
	struct Link {
		double d2;
		size_t from, to;
	};
	std::vector<Link> links;
	// runs of equal planes: [a, b) is plane q, [b, c) the next run
	for (size_t a = 0; a < nPoints;) {
		size_t b = a;
		while (b < nPoints && pts[b].plane == pts[a].plane) { ++b; }
		size_t c = b;
		while (c < nPoints && pts[c].plane == pts[b < nPoints ? b : a].plane) { ++c; }
		if (b < nPoints && pts[b].plane == pts[a].plane + 1) {
			links.clear();
			for (size_t i = a; i < b; ++i) {
				for (size_t j = b; j < c; ++j) {
					const double dx = pts[i].x - pts[j].x, dy = pts[i].y - pts[j].y;
					const double d2 = (dx * dx) + (dy * dy);
					if (d2 <= r2) { links.push_back({d2, i, j}); }
				}
			}
			std::sort(links.begin(), links.end(), [](const Link& u, const Link& v) {
				if (u.d2 != v.d2) { return u.d2 < v.d2; }
				if (u.from != v.from) { return u.from < v.from; }
				return u.to < v.to;
			});
			for (const Link& l : links) {
				if (succ[l.from] == kNone && pred[l.to] == kNone) {
					succ[l.from] = l.to;
					pred[l.to] = l.from;
				}
			}
		}
		a = b;
	}
	size_t next = 1;
	for (size_t k = 0; k < nPoints; ++k) {
		if (pred[k] != kNone) { continue; }
		for (size_t m = k; m != kNone; m = succ[m]) { track[m] = next; }
		++next;
	}
	for (size_t k = 0; k < nPoints; ++k) {
		output[2 * k] = pts[k].id;
		output[2 * k + 1] = track[k];
	}
	return 2 * nPoints;
}


// orc_SplineCoefficients: the coefficient table of a PSF volume [nz][ny][nx] (x fastest) as BSpline3D computes it
// (degree 3, regularisation lambda[3] per axis x, y, z; NULL = none): out receives the reference's layout
// [cell][64] with cells (z, y, x) over (nz - 1) x (ny - 1) x (nx - 1); hdr (optional) the spline's values at the
// voxel centres (step 3). Returns the doubles written, 0 for a dimension below 2.
uint64_t orc_SplineCoefficients(const double* volume, uint64_t nx, uint64_t ny, uint64_t nz, const double* lambda, double* out,
                                double* hdrOut)
{
	if (nx < 2 || ny < 2 || nz < 2) { return 0; }
	const size_t dim[3] = {nx, ny, nz};
	const size_t n = nx * ny * nz;
	std::vector<double> c(volume, volume + n);
	for (int axis = 0; axis < 3; ++axis) {
		std::vector<cplx> poles;
		double gain = 1;
		CubicPoles(lambda ? lambda[axis] : 0.0, poles, gain);
		FilterAxis(c, dim, axis, poles, gain);
	}
	// reflection padding by 1 (dimPadded = dim + 3) and the values at the voxel centres
	const size_t px = nx + 3, py = ny + 3, pz = nz + 3;
	auto refl = [](size_t len, long i) {  // ReflectIndex1D(len, 1) entry i + 1
		const long period = 2 * static_cast<long>(len) - 2;
		const long w = ((i % period) + period) % period;
		return static_cast<size_t>(w < static_cast<long>(len) ? w : period - w);
	};
	std::vector<double> padded(px * py * pz);
	for (size_t z = 0; z < pz; ++z) {
		for (size_t y = 0; y < py; ++y) {
			for (size_t x = 0; x < px; ++x) {
				const size_t src = (refl(nz, static_cast<long>(z) - 1) * ny + refl(ny, static_cast<long>(y) - 1)) * nx + refl(nx, static_cast<long>(x) - 1);
				padded[(z * py + y) * px + x] = c[src];
			}
		}
	}
	std::vector<double> hdr(n);
	for (size_t z = 0; z < nz; ++z) {
		for (size_t y = 0; y < ny; ++y) {
			for (size_t x = 0; x < nx; ++x) {
				// interpolate_at(x + 1, y + 1, z + 1) on the padded coefficients
				const double X = static_cast<double>(x) + 1, Y = static_cast<double>(y) + 1, Z = static_cast<double>(z) + 1;
				const long kx = static_cast<long>(std::floor(X)) - 1, ky = static_cast<long>(std::floor(Y)) - 1,
				           kz = static_cast<long>(std::floor(Z)) - 1;
				double r = 0.0;
				for (long q = 0; q <= 3; ++q) {
					const long iz = kz + q;
					if (iz < 0 || iz >= static_cast<long>(pz)) { continue; }
					const double bz = Bspline3(Z - static_cast<double>(iz));
					for (long i = 0; i <= 3; ++i) {
						const long iy = ky + i;
						if (iy < 0 || iy >= static_cast<long>(py)) { continue; }
						const double byz = Bspline3(Y - static_cast<double>(iy)) * bz;
						for (long j = 0; j <= 3; ++j) {
							const long ix = kx + j;
							if (ix < 0 || ix >= static_cast<long>(px)) { continue; }
							const double bx = Bspline3(X - static_cast<double>(ix));
							r += padded[(static_cast<size_t>(iz) * py + static_cast<size_t>(iy)) * px + static_cast<size_t>(ix)] * bx * byz;
						}
					}
				}
				hdr[(z * ny + y) * nx + x] = r;
			}
		}
	}
	if (hdrOut) { std::copy(hdr.begin(), hdr.end(), hdrOut); }
	// the 64 x 64 system of the monomials at the 1/3 samples, inverted once
	std::vector<double> A(64 * 64), Ai(64 * 64);
	for (int i = 0; i < 4; ++i) {
		const double dx = static_cast<double>(i) / 3.0;
		for (int j = 0; j < 4; ++j) {
			const double dy = static_cast<double>(j) / 3.0;
			for (int k = 0; k < 4; ++k) {
				const double dz = static_cast<double>(k) / 3.0;
				const int row = i * 16 + j * 4 + k;
				for (int l = 0; l < 4; ++l) {
					for (int m = 0; m < 4; ++m) {
						for (int q = 0; q < 4; ++q) {
							A[row * 64 + l * 16 + m * 4 + q] = std::pow(dx, l) * std::pow(dy, m) * std::pow(dz, q);
						}
					}
				}
			}
		}
	}
	if (!InvertGaussJordan(A, Ai, 64)) { return 0; }
	// upsampled values (Upsample by 3 with spline3D on hdr, zeros outside)
	const size_t ux = (nx - 1) * 3 + 1, uy = (ny - 1) * 3 + 1, uz = (nz - 1) * 3 + 1;
	const double step = 1.0 / 3.0;
	auto get = [&](long x, long y, long z) {
		if (x < 0 || x >= static_cast<long>(nx) || y < 0 || y >= static_cast<long>(ny) || z < 0 || z >= static_cast<long>(nz)) { return 0.0; }
		return hdr[(static_cast<size_t>(z) * ny + static_cast<size_t>(y)) * nx + static_cast<size_t>(x)];
	};
	std::vector<double> up(ux * uy * uz);
	for (size_t z = 0; z < uz; ++z) {
		const double pzp = static_cast<double>(z) * step;
		for (size_t y = 0; y < uy; ++y) {
			const double pyp = static_cast<double>(y) * step;
			for (size_t x = 0; x < ux; ++x) {
				const double pxp = static_cast<double>(x) * step;
				const long ix = static_cast<long>(std::floor(pxp)), iy = static_cast<long>(std::floor(pyp)), iz = static_cast<long>(std::floor(pzp));
				double v = 0.0;
				for (long dz = -1; dz <= 2; ++dz) {
					const long Zi = iz + dz;
					const double bz = Bspline3(pzp - static_cast<double>(Zi));
					for (long dy = -1; dy <= 2; ++dy) {
						const long Yi = iy + dy;
						const double byz = Bspline3(pyp - static_cast<double>(Yi)) * bz;
						for (long dx = -1; dx <= 2; ++dx) {
							const long Xi = ix + dx;
							v += get(Xi, Yi, Zi) * (Bspline3(pxp - static_cast<double>(Xi)) * byz);
						}
					}
				}
				up[(z * uy + y) * ux + x] = v;
			}
		}
	}
	const size_t cx = nx - 1, cy = ny - 1, cz = nz - 1;
	size_t base = 0;
	for (size_t z = 0; z < cz; ++z) {
		for (size_t y = 0; y < cy; ++y) {
			for (size_t x = 0; x < cx; ++x, base += 64) {
				double t[64];
				size_t q = 0;
				for (size_t k = 0; k < 4; ++k) {
					for (size_t j = 0; j < 4; ++j) {
						for (size_t i = 0; i < 4; ++i, ++q) { t[q] = up[((z * 3 + k) * uy + (y * 3 + j)) * ux + (x * 3 + i)]; }
					}
				}
				for (size_t i = 0; i < 64; ++i) {
					double acc = 0.0;
					for (size_t j = 0; j < 64; ++j) { acc += Ai[i * 64 + j] * t[j]; }
					out[base + i] = acc;
				}
			}
		}
	}
	return static_cast<uint64_t>(cx * cy * cz * 64);
}

}  // extern "C"
