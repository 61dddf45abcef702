// Gaussian least-squares LM fits (modes 1-4) in FP64 with the reference's exact order of operations, one thread per
// ROI. This file is compiled with -fmad=false: every product and sum is rounded on its own, as in the reference
// built with -ffp-contract=off, so each ROI follows the reference's iteration path decision for decision (sums over
// pixels are sequential in raster order, the damped matrix is inverted by the same equilibrated Gauss-Jordan and
// dp = inverse * beta is accumulated in the same order). Results then differ from the reference only where CUDA's
// exp / sin / cos round differently from the host C library in the last place.
//
// Reference: lib/fit/GaussianFit.cpp:48-295, lib/fit/GaussianModel.cpp:19-52, lib/fit/Fitting.cpp:61-175,
// lib/signal_processing/Matrix.cpp:297-355.
//
// Mapping: thread per candidate, grid-stride. The per-thread normal matrix, its damped copy and the inverse live in
// per-thread local memory (L1-resident); the ROI pixels are re-read through the read-only cache each pass.
#include <algorithm>

#include "pt_common.cuh"

namespace ptb {

namespace {

template <int MODE> struct NpOf;
template <> struct NpOf<kG2Fixed> { static constexpr int v = 4; };
template <> struct NpOf<kG2Sigma> { static constexpr int v = 5; };
template <> struct NpOf<kG3Fixed> { static constexpr int v = 6; };
template <> struct NpOf<kG3Theta> { static constexpr int v = 7; };

template <int MODE>
struct GModel {
	double off, amp, sx, sy, sx2, sy2, c, s, c2, s2, cs;

	__device__ void Make(const double* p, double sigma, double theta)
	{
		off = p[0];
		amp = p[1];
		if constexpr (MODE == kG2Fixed || MODE == kG2Sigma) {
			sx = MODE == kG2Fixed ? sigma : p[4];
			sx2 = sx * sx;
		}
		else {
			const double th = MODE == kG3Fixed ? theta : p[6];
			sx = p[4];
			sy = p[5];
			sx2 = p[4] * p[4];
			sy2 = p[5] * p[5];
			c = cos(th);
			s = sin(th);
			c2 = c * c;
			s2 = s * s;
			cs = c * s;
		}
	}

	template <bool GRAD>
	__device__ __forceinline__ double Eval(double x, double y, double* g) const
	{
		const double X2 = x * x, Y2 = y * y;
		if constexpr (MODE == kG2Fixed || MODE == kG2Sigma) {
			const double e = exp(-(X2 + Y2) / (2 * sx2));
			const double P = amp * e;
			if constexpr (GRAD) {
				g[0] = 1;
				g[1] = e;
				g[2] = P * x / sx2;
				g[3] = P * y / sx2;
				if constexpr (MODE == kG2Sigma) { g[4] = P / (sx * sx2) * (X2 + Y2); }
			}
			return P + off;
		}
		else {
			const double xc = x * c, xs = x * s, yc = y * c, ys = y * s;
			const double f1 = (xc - ys) / sx, f2 = (xs + yc) / sy;
			const double e = exp(-((f1 * f1) + (f2 * f2)));
			const double P = amp * e;
			if constexpr (GRAD) {
				const double xy = x * y, f3 = 2 * xy * cs, f4 = (2 * xy / sx2) - (2 * xy / sy2);
				g[0] = 1;
				g[1] = e;
				g[2] = P * (-(((-2 * c2 * x) + (2 * y * cs)) / sx2) - (((-2 * s2 * x) - (2 * y * cs)) / sy2));
				g[3] = P * ((((2 * s2 * y) - (2 * x * cs)) / sx2) - (((-2 * c2 * y) - (2 * x * cs)) / sy2));
				g[4] = P * (2 * ((xc * xc) - f3 + (ys * ys)) / (sx * sx2));
				g[5] = P * (2 * ((xs * xs) + f3 + (yc * yc)) / (sy * sy2));
				if constexpr (MODE == kG3Theta) { g[6] = P * ((2 * cs * (((X2 - Y2) / sx2) + ((Y2 - X2) / sy2))) - (s2 * f4) + (c2 * f4)); }
			}
			return P + off;
		}
	}
};

// Equilibrated Gauss-Jordan inverse with partial pivoting (Matrix.cpp:297-355); false where the reference throws.
template <int NP>
__device__ bool InvertGJ(double* a, double* inv)
{
	for (int i = 0; i < NP * NP; ++i) { inv[i] = 0.0; }
	for (int i = 0; i < NP; ++i) {
		double scale = 0.0;
		for (int j = 0; j < NP; ++j) {
			const double v = a[i * NP + j];
			if (!isfinite(v)) { return false; }
			scale = fmax(scale, fabs(v));
		}
		if (scale == 0.0) { return false; }
		for (int j = 0; j < NP; ++j) { a[i * NP + j] /= scale; }
		inv[i * NP + i] = 1.0 / scale;
	}
	const double tol = 2.220446049250313e-16 * static_cast<double>(NP);
	for (int i = 0; i < NP; ++i) {
		int piv = i;
		for (int j = i + 1; j < NP; ++j) {
			if (fabs(a[j * NP + i]) > fabs(a[piv * NP + i])) { piv = j; }
		}
		if (!isfinite(a[piv * NP + i]) || fabs(a[piv * NP + i]) <= tol) { return false; }
		if (piv != i) {
			for (int j = 0; j < NP; ++j) {
				const double t = a[i * NP + j];
				a[i * NP + j] = a[piv * NP + j];
				a[piv * NP + j] = t;
				const double u = inv[i * NP + j];
				inv[i * NP + j] = inv[piv * NP + j];
				inv[piv * NP + j] = u;
			}
		}
		const double pinv = 1.0 / a[i * NP + i];
		for (int j = 0; j < NP; ++j) {
			a[i * NP + j] *= pinv;
			inv[i * NP + j] *= pinv;
		}
		for (int j = 0; j < NP; ++j) {
			if (j == i) { continue; }
			const double f = a[j * NP + i];
			for (int k = 0; k < NP; ++k) {
				a[j * NP + k] -= f * a[i * NP + k];
				inv[j * NP + k] -= f * inv[i * NP + k];
			}
		}
	}
	for (int i = 0; i < NP * NP; ++i) {
		if (!isfinite(a[i]) || !isfinite(inv[i])) { return false; }
	}
	return true;
}

__device__ void Store(double* r, int mode, const Cand& c, double x, double y, double off, double amp, double sx, double sy,
                      double th, double qxy)
{
	r[cId] = 0; r[cPlane] = 0; r[cIndex] = 0; r[cChannel] = -1;
	r[cX] = x; r[cY] = y; r[cZ] = 0;
	r[cIntensity] = (amp > kEps && sx > kEps && sy > kEps) ? 2.0 * 3.141592653589793 * amp * sx * sy : -1;
	r[cSigmaX] = sx; r[cSigmaY] = sy; r[cTheta] = th;
	r[cQualityXY] = qxy; r[cQualityZ] = -1;
	r[cAmplitude] = amp; r[cOffset] = off;
	r[cSegIntensity] = c.intensity; r[cSurface] = c.surf;
	r[cCircularity] = (sx > kEps && sy > kEps) ? fmin(sx, sy) / fmax(sx, sy) : 1;
}

template <int MODE>
__device__ void FitExact(const uint16_t* frame, int H, int W, const FitParams& fp, const Cand& cd, double* row)
{
	constexpr int NP = NpOf<MODE>::v;
	auto sentinel = [&](double x, double y) { Store(row, MODE, cd, x, y, -1, -1, -1, -1, -1, -1); };
	const bool nonneg = cd.x >= 0.0 && cd.y >= 0.0;
	const unsigned long long ux = nonneg ? static_cast<unsigned long long>(cd.x) : 0ull;
	const unsigned long long uy = nonneg ? static_cast<unsigned long long>(cd.y) : 0ull;
	const unsigned long long h = static_cast<unsigned long long>(fp.half);
	if (!nonneg || h > ux || ux >= static_cast<unsigned long long>(W) - h || h > uy || uy >= static_cast<unsigned long long>(H) - h) {
		sentinel(cd.x, cd.y);
		return;
	}
	const int roi = fp.roi, n = fp.n, hh = fp.half;
	const uint16_t* base = frame + static_cast<long long>(uy - h) * W + static_cast<long long>(ux - h);
	auto pix = [&](int k, double& X, double& Y) {
		const int i = k / roi, j = k - i * roi;
		X = static_cast<double>(ux + j - hh);
		Y = static_cast<double>(uy + i - hh);
		return static_cast<double>(__ldg(base + static_cast<long long>(i) * W + j));
	};
	double vmin = 1.7976931348623157e308, vmax = -1.7976931348623157e308;
	for (int k = 0; k < n; ++k) {
		double X, Y;
		const double v = pix(k, X, Y);
		vmin = fmin(vmin, v);
		vmax = fmax(vmax, v);
	}
	double lo[NP], p[NP], hi[NP];
	lo[0] = 0; lo[1] = 0; lo[2] = cd.x - 1; lo[3] = cd.y - 1;
	p[0] = vmin; p[1] = vmax - vmin; p[2] = cd.x; p[3] = cd.y;
	hi[0] = 65535; hi[1] = 65535; hi[2] = cd.x + 1; hi[3] = cd.y + 1;
	const double r2 = 1.4142135623730951;
	if constexpr (MODE == kG2Sigma) { lo[4] = 0.1; p[4] = fp.sigmaX; hi[4] = 20; }
	if constexpr (MODE == kG3Fixed || MODE == kG3Theta) {
		lo[4] = lo[5] = 0.1;
		hi[4] = hi[5] = 20;
		p[4] = r2 * fp.sigmaX;
		p[5] = r2 * fp.sigmaY;
	}
	if constexpr (MODE == kG3Theta) { lo[6] = -150; p[6] = fp.theta; hi[6] = 150; }
	double alpha[NP * NP], work[NP * NP], inv[NP * NP], beta[NP], dp[NP], pTry[NP], g[NP];
	GModel<MODE> m;
	auto normal = [&]() {  // GaussianFit.cpp:219-245
		for (int i = 0; i < NP * NP; ++i) { alpha[i] = 0.0; }
		for (int i = 0; i < NP; ++i) { beta[i] = 0.0; }
		double err = 0.0;
		m.Make(p, fp.sigmaX, fp.theta);
		const bool circular = MODE == kG3Theta && fabs(p[4] - p[5]) <= 2.220446049250313e-16;
		for (int k = 0; k < n; ++k) {
			double X, Y;
			const double v = pix(k, X, Y);
			const double hat = m.template Eval<true>(X - p[2], Y - p[3], g);
			const double d = v - hat;
			err += d * d;
			if (circular) { g[NP - 1] = 0.0; }
			for (int a = 0; a < NP; ++a) {
				beta[a] += g[a] * d;
				for (int b = 0; b < NP; ++b) { alpha[a * NP + b] += g[a] * g[b]; }
			}
		}
		return err;
	};
	auto trial = [&]() {  // GaussianFit.cpp:262-271
		GModel<MODE> t;
		t.Make(pTry, fp.sigmaX, fp.theta);
		double res = 0.0;
		for (int k = 0; k < n; ++k) {
			double X, Y;
			const double v = pix(k, X, Y);
			const double d = v - t.template Eval<false>(X - pTry[2], Y - pTry[3], nullptr);
			res += d * d;
		}
		return res;
	};
	auto relStep = [&]() {
		double r = 0.0;
		for (int a = 0; a < NP; ++a) { r = fmax(r, fabs(dp[a]) / fmax(fabs(p[a]), 1e-12)); }
		return r;
	};
	auto maxBeta = [&]() {
		double r = 0.0;
		for (int a = 0; a < NP; ++a) { r = fmax(r, fabs(beta[a])); }
		return r;
	};
	double err = normal();
	bool fin = isfinite(err);
	for (int a = 0; a < NP; ++a) { fin = fin && isfinite(beta[a]); }
	if (!fin) { sentinel(cd.x, cd.y); return; }
	double lambda = 1e-2;
	double mm = maxBeta();
	for (int it = (mm < 1e-6) ? kMaxIter : 0; it < kMaxIter; ++it) {
		for (int i = 0; i < NP * NP; ++i) { work[i] = alpha[i]; }
		for (int i = 0; i < NP; ++i) {
			const int d = i * NP + i;
			work[d] = alpha[d] == 0.0 ? 1.0 : (1.0 + lambda) * alpha[d];
		}
		if (!InvertGJ<NP>(work, inv)) {
			if (lambda < 1e7) { lambda = fmin(lambda * 11, 1e7); continue; }
			sentinel(cd.x, cd.y);
			return;
		}
		for (int i = 0; i < NP; ++i) {
			dp[i] = 0.0;
			for (int j = 0; j < NP; ++j) { dp[i] += inv[i * NP + j] * beta[j]; }
			if (!isfinite(dp[i])) { sentinel(cd.x, cd.y); return; }
			pTry[i] = fmin(fmax(p[i] + dp[i], lo[i]), hi[i]);
		}
		bool tiny = true;
		for (int i = 0; i < NP; ++i) {
			dp[i] = pTry[i] - p[i];
			tiny = tiny && fabs(dp[i]) < 1e-15;
		}
		if (tiny) {
			if (lambda >= 1e7) { break; }
			lambda = fmin(lambda * 11, 1e7);
			continue;
		}
		double quad = 0.0, lin = 0.0;
		for (int i = 0; i < NP; ++i) {
			double t = 0.0;
			for (int j = 0; j < NP; ++j) { t += alpha[i * NP + j] * dp[j]; }
			quad += dp[i] * t;
			lin += dp[i] * beta[i];
		}
		const double gain = (2.0 * lin) - quad;
		if (gain <= 0.0) {
			if (lambda >= 1e7) { break; }
			lambda = fmin(lambda * 11, 1e7);
			if (relStep() < 1e-6 && it >= 2) { break; }
			continue;
		}
		double denom = 0.0;
		for (int i = 0; i < NP; ++i) { denom += dp[i] * ((lambda * dp[i]) + beta[i]); }
		const double errTry = trial();
		const double rho = (err - errTry) / (2.0 * denom);
		if (rho > 1e-2) {
			for (int i = 0; i < NP; ++i) { p[i] = pTry[i]; }
			err = normal();
			lambda = fmax(lambda / 9, 1e-7);
		}
		else {
			if (lambda >= 1e7) { break; }
			lambda = fmin(lambda * 11, 1e7);
		}
		if (it >= 2) {
			if (relStep() < 1e-6) { break; }
			if (err / static_cast<double>(n) < 1e-5) { break; }
			if (maxBeta() < 1e-6) { break; }
		}
	}
	// squared correlation on the model of the last accepted parameters (GaussianFit.cpp:274-295)
	m.Make(p, fp.sigmaX, fp.theta);
	double muD = 0.0, muM = 0.0;
	for (int k = 0; k < n; ++k) {
		double X, Y;
		muD += pix(k, X, Y);
	}
	for (int k = 0; k < n; ++k) {
		double X, Y;
		pix(k, X, Y);
		muM += m.template Eval<false>(X - p[2], Y - p[3], nullptr);
	}
	muD /= static_cast<double>(n);
	muM /= static_cast<double>(n);
	double t1 = 0.0, t2 = 0.0, t3 = 0.0;
	for (int k = 0; k < n; ++k) {
		double X, Y;
		const double d = pix(k, X, Y) - muD;
		t1 += d * (m.template Eval<false>(X - p[2], Y - p[3], nullptr) - muM);
	}
	for (int k = 0; k < n; ++k) {
		double X, Y;
		const double d = pix(k, X, Y) - muD;
		t2 += d * d;
	}
	for (int k = 0; k < n; ++k) {
		double X, Y;
		pix(k, X, Y);
		const double hm = m.template Eval<false>(X - p[2], Y - p[3], nullptr) - muM;
		t3 += hm * hm;
	}
	const double R = t1 / sqrt(t2 * t3);
	const double rr = isnan(R) ? 0 : R * R;
	if (rr < kEps) { sentinel(p[2], p[3]); return; }
	double sx = fp.sigmaX, sy = fp.sigmaY, th = fp.theta;
	if constexpr (MODE == kG2Fixed) { sx = sy = fp.sigmaX; th = 0; }
	if constexpr (MODE == kG2Sigma) { sx = p[4]; sy = sx; th = 0; }
	if constexpr (MODE == kG3Fixed || MODE == kG3Theta) { sx = p[4] / r2; sy = p[5] / r2; }
	if constexpr (MODE == kG3Theta) { th = p[6]; }
	Store(row, MODE, cd, p[2], p[3], p[0], p[1], sx, sy, th, rr);
}

template <int MODE>
__global__ void __launch_bounds__(64) ExactFitKernel(const uint16_t* __restrict__ img, int H, int W, long long N,
                                                     const Cand* __restrict__ cands, const uint32_t* nptr, uint32_t nconst,
                                                     FitParams fp, double* rows, const uint8_t* only)
{
	const uint32_t n = nptr ? *nptr : nconst;
	for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
		if (only && !only[k]) { continue; }
		const Cand cd = cands[k];
		FitExact<MODE>(img + static_cast<long long>(cd.frame) * N, H, W, fp, cd, rows + static_cast<long long>(k) * kCols);
	}
}

}  // namespace

bool LaunchExactFit(const uint16_t* img, int H, int W, long long N, const Cand* cands, const uint32_t* nptr, uint32_t nconst,
                    uint32_t cap, const FitParams& fp, double* rows, const uint8_t* only, cudaStream_t st)
{
	const int threads = 64;
	const uint32_t blocks = std::min<uint32_t>((std::max<uint32_t>(cap, 1) + threads - 1) / threads, 148u * 32u);
	switch (fp.mode) {
		case kG2Fixed: ExactFitKernel<kG2Fixed><<<blocks, threads, 0, st>>>(img, H, W, N, cands, nptr, nconst, fp, rows, only); break;
		case kG2Sigma: ExactFitKernel<kG2Sigma><<<blocks, threads, 0, st>>>(img, H, W, N, cands, nptr, nconst, fp, rows, only); break;
		case kG3Fixed: ExactFitKernel<kG3Fixed><<<blocks, threads, 0, st>>>(img, H, W, N, cands, nptr, nconst, fp, rows, only); break;
		case kG3Theta: ExactFitKernel<kG3Theta><<<blocks, threads, 0, st>>>(img, H, W, N, cands, nptr, nconst, fp, rows, only); break;
		default: return false;
	}
	CountLaunch();
	return PTB_LAUNCHED();
}

}  // namespace ptb
