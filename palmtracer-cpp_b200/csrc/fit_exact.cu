// Gaussian least-squares LM fits (modes 1-4) in FP64 with the reference's exact order of operations, one warp per
// ROI. This file is compiled with -fmad=false: every product and sum is rounded on its own, as in the reference built
// with -ffp-contract=off, so each ROI follows the reference's iteration path decision for decision; results differ
// from the reference only where CUDA's exp / sin / cos round differently from the host C library in the last place.
//
// Reference: lib/fit/GaussianFit.cpp:48-295, lib/fit/GaussianModel.cpp:19-52, lib/fit/Fitting.cpp:61-175,
// lib/signal_processing/Matrix.cpp:297-355.
//
// How the order is kept while the warp works in parallel:
//   * per-pixel terms (model, residual, gradient products) are computed by the lanes, 32 pixels at a time, and staged
//     in shared memory; each accumulator (err, beta[a], alpha[a][b] for a <= b) is then owned by one lane, which adds
//     that chunk's terms in pixel order - the reference's sequential sums, term for term;
//   * the damped matrix is inverted column-parallel: lane c < p owns column c of the matrix, lane p + c column c of
//     the inverse, and every element goes through exactly the reference's Gauss-Jordan operations (equilibration,
//     partial pivoting, row normalisation, elimination), whose results do not depend on the order across elements;
//   * dp = inverse * beta and every other small-vector step run identically on all lanes in the reference's order.
#include <algorithm>

#include "pt_common.cuh"

namespace ptb {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarps = 4;
constexpr int kMaxTerms = 36;  // 1 + 7 + 28 for mode 4

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

struct WarpSmem {
	double terms[kMaxTerms][33];  // [accumulator][pixel of the chunk], padded
	double acc[kMaxTerms + 4];    // broadcast of the accumulators
};

struct Roi {
	const uint16_t* base;
	int W, roi, n, half;
	unsigned long long ux, uy;
	__device__ __forceinline__ double Pix(int k, double& X, double& Y) const
	{
		const int i = k / roi, j = k - i * roi;
		X = static_cast<double>(ux + j - half);
		Y = static_cast<double>(uy + i - half);
		return static_cast<double>(__ldg(base + static_cast<long long>(i) * W + j));
	}
};

// err, beta and alpha (upper triangle, row major) at p, summed in pixel order. Every lane returns the same values.
template <int MODE>
__device__ double NormalExact(WarpSmem& S, const Roi& R, const GModel<MODE>& m, const double* p, bool circular,
                              double (&beta)[NpOf<MODE>::v], double (&alphaU)[NpOf<MODE>::v * (NpOf<MODE>::v + 1) / 2])
{
	constexpr int NP = NpOf<MODE>::v;
	constexpr int NT = 1 + NP + NP * (NP + 1) / 2;
	const int lane = threadIdx.x & 31;
	double acc0 = 0.0, acc1 = 0.0;  // accumulators lane and lane + 32
	for (int c0 = 0; c0 < R.n; c0 += 32) {
		const int k = c0 + lane;
		if (k < R.n) {
			double X, Y, g[NP];
			const double v = R.Pix(k, X, Y);
			const double hat = m.template Eval<true>(X - p[2], Y - p[3], g);
			const double d = v - hat;
			if (circular) { g[NP - 1] = 0.0; }
			S.terms[0][lane] = d * d;
			#pragma unroll
			for (int a = 0; a < NP; ++a) { S.terms[1 + a][lane] = g[a] * d; }
			int q = 1 + NP;
			#pragma unroll
			for (int a = 0; a < NP; ++a) {
				#pragma unroll
				for (int b = a; b < NP; ++b) { S.terms[q++][lane] = g[a] * g[b]; }
			}
		}
		__syncwarp();
		const int cnt = min(32, R.n - c0);
		if (lane < NT) {
			for (int j = 0; j < cnt; ++j) { acc0 += S.terms[lane][j]; }
		}
		if (lane + 32 < NT) {
			for (int j = 0; j < cnt; ++j) { acc1 += S.terms[lane + 32][j]; }
		}
		__syncwarp();
	}
	if (lane < NT) { S.acc[lane] = acc0; }
	if (lane + 32 < NT) { S.acc[lane + 32] = acc1; }
	__syncwarp();
	const double err = S.acc[0];
	#pragma unroll
	for (int a = 0; a < NP; ++a) { beta[a] = S.acc[1 + a]; }
	#pragma unroll
	for (int q = 0; q < NP * (NP + 1) / 2; ++q) { alphaU[q] = S.acc[1 + NP + q]; }
	__syncwarp();
	return err;
}

template <int NP>
__device__ __forceinline__ int U(int a, int b) { return a <= b ? a * NP - (a * (a - 1)) / 2 + (b - a) : b * NP - (b * (b - 1)) / 2 + (a - b); }

// Column-parallel equilibrated Gauss-Jordan inverse of the damped matrix, then dp = inverse * beta in the reference's
// order (Matrix.cpp:297-355, GaussianFit.cpp:85-106). Returns false where the reference's inversion throws.
template <int NP>
__device__ bool SolveExact(const double (&alphaU)[NP * (NP + 1) / 2], const double (&beta)[NP], double lambda, double (&dp)[NP])
{
	const int lane = threadIdx.x & 31;
	const bool isA = lane < NP, isI = lane >= NP && lane < 2 * NP;
	const int col = isA ? lane : lane - NP;
	double cv[NP];
	bool fin = true;
	#pragma unroll
	for (int r = 0; r < NP; ++r) {
		double v = 0.0;
		if (isA) {
			const double a = alphaU[U<NP>(r, col)];
			v = r == col ? (a == 0.0 ? 1.0 : (1.0 + lambda) * a) : a;
			fin = fin && isfinite(v);
		}
		cv[r] = v;
	}
	if (!__all_sync(kFull, fin)) { return false; }
	// row equilibration: scale_r = max_c |a[r][c]| (order-independent), in /= scale, out[r][r] = 1 / scale
	#pragma unroll
	for (int r = 0; r < NP; ++r) {
		double m = isA ? fabs(cv[r]) : 0.0;
		#pragma unroll
		for (int d = 16; d > 0; d >>= 1) { m = fmax(m, __shfl_xor_sync(kFull, m, d)); }
		if (m == 0.0) { return false; }
		if (isA) { cv[r] /= m; }
		if (isI) { cv[r] = r == col ? 1.0 / m : 0.0; }
	}
	const double tol = 2.220446049250313e-16 * static_cast<double>(NP);
	#pragma unroll
	for (int i = 0; i < NP; ++i) {
		int piv = i;
		double best = cv[i];
		#pragma unroll
		for (int j = i + 1; j < NP; ++j) {
			if (fabs(cv[j]) > fabs(best)) { piv = j; best = cv[j]; }
		}
		piv = __shfl_sync(kFull, piv, i);
		best = __shfl_sync(kFull, best, i);
		if (!isfinite(best) || fabs(best) <= tol) { return false; }
		if (piv != i) {
			#pragma unroll
			for (int j = i + 1; j < NP; ++j) {
				if (j == piv) {
					const double t = cv[i];
					cv[i] = cv[j];
					cv[j] = t;
				}
			}
		}
		const double pinv = 1.0 / __shfl_sync(kFull, cv[i], i);
		cv[i] *= pinv;
		#pragma unroll
		for (int j = 0; j < NP; ++j) {
			if (j == i) { continue; }
			const double f = __shfl_sync(kFull, cv[j], i);
			cv[j] -= f * cv[i];
		}
	}
	fin = true;
	#pragma unroll
	for (int r = 0; r < NP; ++r) { fin = fin && ((!isA && !isI) || isfinite(cv[r])); }
	if (!__all_sync(kFull, fin)) { return false; }
	// dp_i = sum_j inv[i][j] beta_j, j ascending; column j of the inverse is on lane NP + j
	#pragma unroll
	for (int i = 0; i < NP; ++i) {
		double s = 0.0;
		#pragma unroll
		for (int j = 0; j < NP; ++j) { s += __shfl_sync(kFull, cv[i], NP + j) * beta[j]; }
		dp[i] = s;
	}
	return true;
}

__device__ void StoreRow(double* row, const Cand& c, double x, double y, double off, double amp, double sx, double sy,
                         double th, double qxy)
{
	const int lane = threadIdx.x & 31;
	double v;
	switch (lane) {
		case cChannel: v = -1; break;
		case cX: v = x; break;
		case cY: v = y; break;
		case cIntensity: v = (amp > kEps && sx > kEps && sy > kEps) ? 2.0 * 3.141592653589793 * amp * sx * sy : -1; break;
		case cSigmaX: v = sx; break;
		case cSigmaY: v = sy; break;
		case cTheta: v = th; break;
		case cQualityXY: v = qxy; break;
		case cQualityZ: v = -1; break;
		case cAmplitude: v = amp; break;
		case cOffset: v = off; break;
		case cSegIntensity: v = c.intensity; break;
		case cSurface: v = c.surf; break;
		case cCircularity: v = (sx > kEps && sy > kEps) ? fmin(sx, sy) / fmax(sx, sy) : 1; break;
		default: v = 0; break;
	}
	if (lane < kCols) { row[lane] = v; }
}

// Sum of the lanes' per-pixel values over the ROI in pixel order (lane 0 of each chunk first).
__device__ double ChunkedOrderedSum(WarpSmem& S, double mine, int cnt, double total)
{
	const int lane = threadIdx.x & 31;
	S.terms[0][lane] = mine;
	__syncwarp();
	if (lane == 0) {
		for (int j = 0; j < cnt; ++j) { total += S.terms[0][j]; }
		S.acc[0] = total;
	}
	__syncwarp();
	total = S.acc[0];
	__syncwarp();
	return total;
}

template <int MODE>
__device__ void FitWarp(WarpSmem& S, const uint16_t* frame, int H, int W, const FitParams& fp, const Cand& cd, double* row)
{
	constexpr int NP = NpOf<MODE>::v;
	constexpr int NU = NP * (NP + 1) / 2;
	const int lane = threadIdx.x & 31;
	auto sentinel = [&](double x, double y) { StoreRow(row, cd, x, y, -1, -1, -1, -1, -1, -1); };
	const bool nonneg = cd.x >= 0.0 && cd.y >= 0.0;
	const unsigned long long ux = nonneg ? static_cast<unsigned long long>(cd.x) : 0ull;
	const unsigned long long uy = nonneg ? static_cast<unsigned long long>(cd.y) : 0ull;
	const unsigned long long h = static_cast<unsigned long long>(fp.half);
	if (!nonneg || h > ux || ux >= static_cast<unsigned long long>(W) - h || h > uy || uy >= static_cast<unsigned long long>(H) - h) {
		sentinel(cd.x, cd.y);
		return;
	}
	Roi R;
	R.base = frame + static_cast<long long>(uy - h) * W + static_cast<long long>(ux - h);
	R.W = W;
	R.roi = fp.roi;
	R.n = fp.n;
	R.half = fp.half;
	R.ux = ux;
	R.uy = uy;
	double vmin = 1.7976931348623157e308, vmax = -1.7976931348623157e308;
	for (int k = lane; k < R.n; k += 32) {
		double X, Y;
		const double v = R.Pix(k, X, Y);
		vmin = fmin(vmin, v);
		vmax = fmax(vmax, v);
	}
	#pragma unroll
	for (int d = 16; d > 0; d >>= 1) {
		vmin = fmin(vmin, __shfl_xor_sync(kFull, vmin, d));
		vmax = fmax(vmax, __shfl_xor_sync(kFull, vmax, d));
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
	double alphaU[NU], beta[NP], dp[NP], pTry[NP];
	GModel<MODE> m;
	auto normal = [&]() {
		m.Make(p, fp.sigmaX, fp.theta);
		const bool circular = MODE == kG3Theta && fabs(p[4] - p[5]) <= 2.220446049250313e-16;
		return NormalExact<MODE>(S, R, m, p, circular, beta, alphaU);
	};
	auto trial = [&]() {
		GModel<MODE> t;
		t.Make(pTry, fp.sigmaX, fp.theta);
		double res = 0.0;
		for (int c0 = 0; c0 < R.n; c0 += 32) {
			const int k = c0 + lane;
			double sq = 0.0;
			if (k < R.n) {
				double X, Y;
				const double v = R.Pix(k, X, Y);
				const double d = v - t.template Eval<false>(X - pTry[2], Y - pTry[3], nullptr);
				sq = d * d;
			}
			res = ChunkedOrderedSum(S, sq, min(32, R.n - c0), res);
		}
		return res;
	};
	auto relStep = [&]() {
		double r = 0.0;
		#pragma unroll
		for (int a = 0; a < NP; ++a) { r = fmax(r, fabs(dp[a]) / fmax(fabs(p[a]), 1e-12)); }
		return r;
	};
	auto maxBeta = [&]() {
		double r = 0.0;
		#pragma unroll
		for (int a = 0; a < NP; ++a) { r = fmax(r, fabs(beta[a])); }
		return r;
	};
	double err = normal();
	bool fin = isfinite(err);
	#pragma unroll
	for (int a = 0; a < NP; ++a) { fin = fin && isfinite(beta[a]); }
	if (!fin) { sentinel(cd.x, cd.y); return; }
	double lambda = 1e-2;
	const double mm = maxBeta();
	for (int it = (mm < 1e-6) ? kMaxIter : 0; it < kMaxIter; ++it) {
		if (!SolveExact<NP>(alphaU, beta, lambda, dp)) {
			if (lambda < 1e7) { lambda = fmin(lambda * 11, 1e7); continue; }
			sentinel(cd.x, cd.y);
			return;
		}
		bool dpFin = true;
		#pragma unroll
		for (int i = 0; i < NP; ++i) {
			dpFin = dpFin && isfinite(dp[i]);
			pTry[i] = fmin(fmax(p[i] + dp[i], lo[i]), hi[i]);
		}
		if (!dpFin) { sentinel(cd.x, cd.y); return; }
		bool tiny = true;
		#pragma unroll
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
		#pragma unroll
		for (int i = 0; i < NP; ++i) {
			double t = 0.0;
			#pragma unroll
			for (int j = 0; j < NP; ++j) { t += alphaU[U<NP>(i, j)] * dp[j]; }
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
		#pragma unroll
		for (int i = 0; i < NP; ++i) { denom += dp[i] * ((lambda * dp[i]) + beta[i]); }
		const double errTry = trial();
		const double rho = (err - errTry) / (2.0 * denom);
		if (rho > 1e-2) {
			#pragma unroll
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
			if (err / static_cast<double>(R.n) < 1e-5) { break; }
			if (maxBeta() < 1e-6) { break; }
		}
	}
	// squared correlation on the model of the last accepted parameters (GaussianFit.cpp:274-295)
	m.Make(p, fp.sigmaX, fp.theta);
	double muD = 0.0, muM = 0.0;
	for (int c0 = 0; c0 < R.n; c0 += 32) {
		const int k = c0 + lane;
		double v = 0.0;
		if (k < R.n) {
			double X, Y;
			v = R.Pix(k, X, Y);
		}
		muD = ChunkedOrderedSum(S, v, min(32, R.n - c0), muD);
	}
	for (int c0 = 0; c0 < R.n; c0 += 32) {
		const int k = c0 + lane;
		double hv = 0.0;
		if (k < R.n) {
			double X, Y;
			R.Pix(k, X, Y);
			hv = m.template Eval<false>(X - p[2], Y - p[3], nullptr);
		}
		muM = ChunkedOrderedSum(S, hv, min(32, R.n - c0), muM);
	}
	muD /= static_cast<double>(R.n);
	muM /= static_cast<double>(R.n);
	double t1 = 0.0, t2 = 0.0, t3 = 0.0;
	for (int c0 = 0; c0 < R.n; c0 += 32) {
		const int k = c0 + lane;
		double a = 0.0, b = 0.0, c = 0.0;
		if (k < R.n) {
			double X, Y;
			const double d = R.Pix(k, X, Y) - muD;
			const double hm = m.template Eval<false>(X - p[2], Y - p[3], nullptr) - muM;
			a = d * hm;
			b = d * d;
			c = hm * hm;
		}
		const int cnt = min(32, R.n - c0);
		S.terms[0][lane] = a;
		S.terms[1][lane] = b;
		S.terms[2][lane] = c;
		__syncwarp();
		if (lane < 3) {
			double acc = lane == 0 ? t1 : lane == 1 ? t2 : t3;
			for (int j = 0; j < cnt; ++j) { acc += S.terms[lane][j]; }
			S.acc[lane] = acc;
		}
		__syncwarp();
		t1 = S.acc[0];
		t2 = S.acc[1];
		t3 = S.acc[2];
		__syncwarp();
	}
	const double Rr = t1 / sqrt(t2 * t3);
	const double rr = isnan(Rr) ? 0 : Rr * Rr;
	if (rr < kEps) { sentinel(p[2], p[3]); return; }
	double sx = fp.sigmaX, sy = fp.sigmaY, th = fp.theta;
	if constexpr (MODE == kG2Fixed) { sx = sy = fp.sigmaX; th = 0; }
	if constexpr (MODE == kG2Sigma) { sx = p[4]; sy = sx; th = 0; }
	if constexpr (MODE == kG3Fixed || MODE == kG3Theta) { sx = p[4] / r2; sy = p[5] / r2; }
	if constexpr (MODE == kG3Theta) { th = p[6]; }
	StoreRow(row, cd, p[2], p[3], p[0], p[1], sx, sy, th, rr);
}

template <int MODE>
__global__ void __launch_bounds__(32 * kWarps) ExactFitKernel(const uint16_t* __restrict__ img, int H, int W, long long N,
                                                              const Cand* __restrict__ cands, const uint32_t* nptr,
                                                              uint32_t nconst, FitParams fp, double* rows, const uint8_t* only)
{
	__shared__ WarpSmem smem[kWarps];
	WarpSmem& S = smem[threadIdx.x >> 5];
	const uint32_t n = nptr ? *nptr : nconst;
	const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
	for (uint32_t k = warp; k < n; k += nw) {
		if (only && !only[k]) { continue; }
		const Cand cd = cands[k];
		FitWarp<MODE>(S, img + static_cast<long long>(cd.frame) * N, H, W, fp, cd, rows + static_cast<long long>(k) * kCols);
	}
}

}  // namespace

bool LaunchExactFit(const uint16_t* img, int H, int W, long long N, const Cand* cands, const uint32_t* nptr, uint32_t nconst,
                    uint32_t cap, const FitParams& fp, double* rows, const uint8_t* only, cudaStream_t st)
{
	const uint32_t blocks = std::min<uint32_t>((std::max<uint32_t>(cap, 1) + kWarps - 1) / kWarps, 148u * 16u);
	switch (fp.mode) {
		case kG2Fixed: ExactFitKernel<kG2Fixed><<<blocks, 32 * kWarps, 0, st>>>(img, H, W, N, cands, nptr, nconst, fp, rows, only); break;
		case kG2Sigma: ExactFitKernel<kG2Sigma><<<blocks, 32 * kWarps, 0, st>>>(img, H, W, N, cands, nptr, nconst, fp, rows, only); break;
		case kG3Fixed: ExactFitKernel<kG3Fixed><<<blocks, 32 * kWarps, 0, st>>>(img, H, W, N, cands, nptr, nconst, fp, rows, only); break;
		case kG3Theta: ExactFitKernel<kG3Theta><<<blocks, 32 * kWarps, 0, st>>>(img, H, W, N, cands, nptr, nconst, fp, rows, only); break;
		default: return false;
	}
	CountLaunch();
	return PTB_LAUNCHED();
}

}  // namespace ptb
