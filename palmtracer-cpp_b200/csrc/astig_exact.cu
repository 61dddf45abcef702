// z from fitted widths with the astigmatism model (the reference's Astigmatism3DEstimation export, CPU/main.cpp:324-353
// -> AstigFit::Estimate, lib/fit/AstigFit.cpp:36-59): one thread per point runs the 201-point grid of the squared width
// error over [-zMax, zMax], Brent's minimisation on the best grid point +-2 steps (:342-447, constants
// AstigFit.hpp:110-114), keeps the grid point when Brent does not improve on it, and scores the widths' compatibility
// (:99-109). Every step is an IEEE basic operation or a square root, both correctly rounded on the GPU; compiled
// without FMA contraction (as the reference is), the result equals the reference's bit for bit. min/max are written
// as the comparisons std::min/std::max make, so NaN widths take the same path.
#include <algorithm>

#include "pt_common.cuh"

namespace ptb {

namespace {

struct AstigAxis {
	double z0, w, c3, c4, a;
};

struct AstigModel {
	AstigAxis x, y;
	double scale;  // 1 / pixel size (widths in nm -> px)
};

__device__ __forceinline__ double Width(const AstigAxis& m, double scale, double z)
{
	const double u = (z - m.z0) / m.w;
	const double u2 = u * u, u3 = u2 * u, u4 = u3 * u;
	const double poly = 1.0 + u2 + (m.c3 * u3) + (m.c4 * u4);
	const double p = 0.0 < poly ? poly : 0.0;
	return scale * (m.a * sqrt(p));
}

__device__ __forceinline__ double WidthError(const AstigModel& m, double z, double sx, double sy)
{
	const double dx = Width(m.x, m.scale, z) - sx, dy = Width(m.y, m.scale, z) - sy;
	return (dx * dx) + (dy * dy);
}

__device__ __forceinline__ double MaxOf(double a, double b) { return a < b ? b : a; }
__device__ __forceinline__ double MinOf(double a, double b) { return b < a ? b : a; }

__global__ void AstigEstimateKernel(const double* __restrict__ in, double* __restrict__ out, uint64_t n, AstigModel m, double zMax)
{
	constexpr int kGrid = 201, kIter = 80;
	constexpr double kTol = 1e-3, kZTol = 1e-9, kQ = 0.2, kGold = 1.0 - 0.6180339887498948482;
	const double lo = -zMax, hi = zMax, span = hi - lo;
	for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
		const double sx = in[2 * i], sy = in[2 * i + 1];
		double bestZ = lo, bestE = __longlong_as_double(0x7ff0000000000000ll);  // +inf
		for (int g = 0; g < kGrid; ++g) {
			const double z = lo + ((static_cast<double>(g) / static_cast<double>(kGrid - 1)) * span);
			const double e = WidthError(m, z, sx, sy);
			if (e < bestE) {
				bestE = e;
				bestZ = z;
			}
		}
		const double step = span / static_cast<double>(kGrid - 1);
		double a = MaxOf(lo, MinOf(bestZ - (2.0 * step), hi));
		double b = MaxOf(lo, MinOf(bestZ + (2.0 * step), hi));
		if (b < a) {
			const double t = a;
			a = b;
			b = t;
		}
		// x: best point, w: second best, v: previous w; d: last step, e: the step before it
		double x = a + (kGold * (b - a)), w = x, v = x;
		double fx = WidthError(m, x, sx, sy), fw = fx, fv = fx, d = 0.0, e = 0.0;
		for (int it = 0; it < kIter; ++it) {
			const double mid = 0.5 * (a + b);
			const double tol1 = (kTol * fabs(x)) + 1e-12, tol2 = 2.0 * tol1;
			if (fabs(x - mid) <= tol2 - (0.5 * (b - a))) { break; }
			bool para = false;
			if (fabs(e) > tol1) {
				const double r = (x - w) * (fx - fv);
				double q = (x - v) * (fx - fw);
				double p = ((x - v) * q) - ((x - w) * r);
				q = 2.0 * (q - r);
				if (q > 0.0) { p = -p; }
				q = fabs(q);
				const double eOld = e;
				e = d;
				if (fabs(p) < fabs(0.5 * q * eOld) && p > q * (a - x) && p < q * (b - x)) {
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
			const double u = x + (fabs(d) >= tol1 ? d : (d > 0.0 ? tol1 : -tol1));
			const double fu = WidthError(m, u, sx, sy);
			if (fu <= fx) {
				if (u < x) { b = x; }
				else { a = x; }
				v = w; fv = fw; w = x; fw = fx; x = u; fx = fu;
			}
			else {
				if (u < x) { a = u; }
				else { b = u; }
				if (fu <= fw || fabs(x - w) <= kZTol) { v = w; fv = fw; w = u; fw = fu; }
				else if (fu <= fv || fabs(v - x) <= kZTol || fabs(v - w) <= kZTol) { v = u; fv = fu; }
			}
		}
		const double z = fx < bestE ? x : bestZ;
		const double px = Width(m.x, m.scale, z), py = Width(m.y, m.scale, z);
		double score = 0.0;
		if (isfinite(px) && isfinite(py) && px > 0 && py > 0 && isfinite(sx) && isfinite(sy) && sx > 0 && sy > 0) {
			const double rx = (sx - px) / px / kQ, ry = (sy - py) / py / kQ;
			score = 1.0 / (1.0 + (0.5 * ((rx * rx) + (ry * ry))));
		}
		out[2 * i] = z;
		out[2 * i + 1] = score;
	}
}

}  // namespace

// dIn, dOut: device [n][2]; model [z0, w, c3, c4, A] for x then y (host).
bool LaunchAstigEstimate(const double* dIn, double* dOut, uint64_t n, double pixelSize, const double* model, double zMax, cudaStream_t st)
{
	if (n == 0) { return true; }
	AstigModel m;
	m.x = {model[0], model[1], model[2], model[3], model[4]};
	m.y = {model[5], model[6], model[7], model[8], model[9]};
	m.scale = 1.0 / pixelSize;
	const uint64_t blocks = std::min<uint64_t>((n + 127) / 128, 148ull * 16);
	AstigEstimateKernel<<<static_cast<unsigned>(blocks), 128, 0, st>>>(dIn, dOut, n, m, zMax);
	CountLaunch();
	return PTB_LAUNCHED();
}

}  // namespace ptb
