// Per-ROI Gaussian least-squares Levenberg-Marquardt fits (modes 1-4), one warp per ROI.
//
// Reference: lib/fit/GaussianFit.cpp:48-295 (LM loop, gain, trial error, R^2), lib/fit/GaussianModel.cpp:19-52
// (model and gradient), lib/fit/Fitting.cpp:61-175 (ROI gather, initial parameters, bounds, output row) and
// lib/signal_processing/Matrix.cpp:297-355 (equilibrated Gauss-Jordan with partial pivoting).
//
// Mapping: the 32 lanes of a warp own the ROI pixels (idx = lane + 32 k). The normal equations J^T J, J^T r and the
// residual are warp all-reduced with an XOR butterfly, which leaves bitwise-identical sums on every lane, so the
// small-matrix part of the iteration and every accept/reject decision run redundantly and uniformly on all lanes.
// The damped system is solved column-parallel: lane c < p holds column c, lane p the right-hand side. Parameters are
// kept in ROI-local coordinates (origin at the integer candidate position) so that FP32 does not lose the sub-pixel
// part of large image coordinates.
#include <algorithm>

#include "pt_common.cuh"

namespace ptb {

namespace {

constexpr unsigned kFull = 0xffffffffu;

template <int MODE> struct Np;
template <> struct Np<kG2Fixed> { static constexpr int v = 4; };
template <> struct Np<kG2Sigma> { static constexpr int v = 5; };
template <> struct Np<kG3Fixed> { static constexpr int v = 6; };
template <> struct Np<kG3Theta> { static constexpr int v = 7; };

template <typename T> __device__ __forceinline__ T Exp(T x);
template <> __device__ __forceinline__ double Exp<double>(double x) { return exp(x); }
template <> __device__ __forceinline__ float Exp<float>(float x) { return expf(x); }

template <typename T> __device__ __forceinline__ bool Finite(T x) { return isfinite(x); }

template <typename T> __device__ __forceinline__ T WarpSum(T v)
{
	#pragma unroll
	for (int d = 16; d > 0; d >>= 1) { v += __shfl_xor_sync(kFull, v, d); }
	return v;
}
template <typename T> __device__ __forceinline__ T WarpMin(T v)
{
	#pragma unroll
	for (int d = 16; d > 0; d >>= 1) { v = min(v, __shfl_xor_sync(kFull, v, d)); }
	return v;
}
template <typename T> __device__ __forceinline__ T WarpMax(T v)
{
	#pragma unroll
	for (int d = 16; d > 0; d >>= 1) { v = max(v, __shfl_xor_sync(kFull, v, d)); }
	return v;
}

// Gaussian PSF at offset (x, y) from its centre, with its gradient (GaussianModel.cpp:19-52). Anisotropic modes use
// the reference's sqrt(2)*sigma convention: exp(-(F1^2 + F2^2)).
template <typename T, int MODE>
struct Model {
	T off, amp, sx, sx2, sy, sy2, c, s, c2, s2, cs;

	__device__ void Make(const T* p, T sigma, T theta)
	{
		off = p[0];
		amp = p[1];
		if constexpr (MODE == kG2Fixed || MODE == kG2Sigma) {
			sx = MODE == kG2Fixed ? sigma : p[4];
			sx2 = sx * sx;
		}
		else {
			const T th = MODE == kG3Fixed ? theta : p[6];
			sx = p[4];
			sy = p[5];
			sx2 = sx * sx;
			sy2 = sy * sy;
			c = cos(th);
			s = sin(th);
			c2 = c * c;
			s2 = s * s;
			cs = c * s;
		}
	}

	template <bool GRAD>
	__device__ __forceinline__ T Eval(T x, T y, T* g) const
	{
		const T X2 = x * x, Y2 = y * y;
		if constexpr (MODE == kG2Fixed || MODE == kG2Sigma) {
			const T e = Exp<T>(-(X2 + Y2) / (T(2) * sx2));
			const T P = amp * e;
			if constexpr (GRAD) {
				g[0] = T(1);
				g[1] = e;
				g[2] = P * x / sx2;
				g[3] = P * y / sx2;
				if constexpr (MODE == kG2Sigma) { g[4] = P / (sx * sx2) * (X2 + Y2); }
			}
			return P + off;
		}
		else {
			const T xc = x * c, xs = x * s, yc = y * c, ys = y * s;
			const T f1 = (xc - ys) / sx, f2 = (xs + yc) / sy;
			const T e = Exp<T>(-((f1 * f1) + (f2 * f2)));
			const T P = amp * e;
			if constexpr (GRAD) {
				const T xy = x * y, f3 = T(2) * xy * cs, f4 = (T(2) * xy / sx2) - (T(2) * xy / sy2);
				g[0] = T(1);
				g[1] = e;
				g[2] = P * (-(((T(-2) * c2 * x) + (T(2) * y * cs)) / sx2) - (((T(-2) * s2 * x) - (T(2) * y * cs)) / sy2));
				g[3] = P * ((((T(2) * s2 * y) - (T(2) * x * cs)) / sx2) - (((T(-2) * c2 * y) - (T(2) * x * cs)) / sy2));
				g[4] = P * (T(2) * ((xc * xc) - f3 + (ys * ys)) / (sx * sx2));
				g[5] = P * (T(2) * ((xs * xs) + f3 + (yc * yc)) / (sy * sy2));
				if constexpr (MODE == kG3Theta) {
					g[6] = P * ((T(2) * cs * (((X2 - Y2) / sx2) + ((Y2 - X2) / sy2))) - (s2 * f4) + (c2 * f4));
				}
			}
			return P + off;
		}
	}
};

// Output row (Fitting.cpp:61-106), written by lanes 0..17 (one column each).
__device__ void StoreRow(double* row, int mode, double segI, double surf, double x, double y, double z, double offset,
                         double amp, double sx, double sy, double theta, double qxy, double qz)
{
	const int lane = threadIdx.x & 31;
	double v[kCols];
	v[cId] = 0; v[cPlane] = 0; v[cIndex] = 0; v[cChannel] = -1;
	v[cX] = x; v[cY] = y; v[cZ] = z;
	if (mode == kNone) { v[cIntensity] = segI; }
	else if (mode == kSplineEmccd) { v[cIntensity] = amp; }
	else {
		// left-to-right product as in the reference: ((2 pi) A) sx sy
		v[cIntensity] = (amp > kEps && sx > kEps && sy > kEps) ? __dmul_rn(__dmul_rn(__dmul_rn(2.0 * 3.141592653589793, amp), sx), sy) : -1.0;
	}
	v[cSigmaX] = sx; v[cSigmaY] = sy; v[cTheta] = theta;
	v[cQualityXY] = qxy; v[cQualityZ] = qz;
	v[cAmplitude] = amp; v[cOffset] = offset;
	v[cSegIntensity] = segI; v[cSurface] = surf;
	v[cCircularity] = (sx > kEps && sy > kEps) ? fmin(sx, sy) / fmax(sx, sy) : 1.0;
	#pragma unroll
	for (int c = 0; c < kCols; ++c) {
		if (lane == c) { row[c] = v[c]; }
	}
}

// Column-parallel solve of (alpha with damped diagonal) dp = beta; false where InverseGaussJordan throws.
template <typename T, int NP>
__device__ bool Solve(const T (&alpha)[NP][NP], const T (&beta)[NP], T lambda, T (&dp)[NP])
{
	const int lane = threadIdx.x & 31;
	T col[NP];
	bool ok = true;
	// row equilibration (every lane computes every row scale from its full copy)
	T scale[NP];
	#pragma unroll
	for (int r = 0; r < NP; ++r) {
		T sc = T(0);
		#pragma unroll
		for (int c = 0; c < NP; ++c) {
			const T a = r == c ? (alpha[r][c] == T(0) ? T(1) : (T(1) + lambda) * alpha[r][c]) : alpha[r][c];
			ok = ok && Finite(a);
			sc = max(sc, fabs(a));
		}
		ok = ok && sc != T(0);
		scale[r] = sc;
	}
	if (!ok) { return false; }
	#pragma unroll
	for (int r = 0; r < NP; ++r) {
		T v = T(0);
		#pragma unroll
		for (int c = 0; c < NP; ++c) {
			if (lane == c) { v = r == c ? (alpha[r][c] == T(0) ? T(1) : (T(1) + lambda) * alpha[r][c]) : alpha[r][c]; }
		}
		if (lane == NP) { v = beta[r]; }
		col[r] = v / scale[r];
	}
	const T tol = (sizeof(T) == 8 ? T(2.220446049250313e-16) : T(1.1920929e-07)) * T(NP);
	#pragma unroll
	for (int i = 0; i < NP; ++i) {
		// partial pivot on column i (lane i), first maximum in row order
		int piv = i;
		T best = fabs(col[i]);
		#pragma unroll
		for (int r = i + 1; r < NP; ++r) {
			if (fabs(col[r]) > best) { best = fabs(col[r]); piv = r; }
		}
		piv = __shfl_sync(kFull, piv, i);
		T pv = col[i];
		#pragma unroll
		for (int r = i + 1; r < NP; ++r) {
			if (r == piv) { pv = col[r]; }
		}
		pv = __shfl_sync(kFull, pv, i);
		if (!Finite(pv) || fabs(pv) <= tol) { return false; }
		if (piv != i) {
			#pragma unroll
			for (int r = i + 1; r < NP; ++r) {
				if (r == piv) {
					const T t = col[i];
					col[i] = col[r];
					col[r] = t;
				}
			}
		}
		const T pinv = T(1) / pv;
		col[i] *= pinv;
		#pragma unroll
		for (int j = 0; j < NP; ++j) {
			if (j == i) { continue; }
			const T f = __shfl_sync(kFull, col[j], i);
			col[j] -= f * col[i];
		}
	}
	bool fin = true;
	#pragma unroll
	for (int r = 0; r < NP; ++r) { fin = fin && Finite(col[r]); }
	fin = __all_sync(kFull, fin || lane > NP);
	#pragma unroll
	for (int r = 0; r < NP; ++r) { dp[r] = __shfl_sync(kFull, col[r], NP); }
	return fin;
}

template <typename T, int MODE>
struct Roi {
	const uint16_t* base;  // pixel (0, 0) of the ROI
	int W, roi, n;
	T x0;                  // local coordinate of ROI column 0 (= -half)
};

// Sum over the ROI of model/gradient products: err, beta, alpha (upper triangle mirrored). Returns err.
template <typename T, int MODE>
__device__ T NormalEquations(const Roi<T, MODE>& R, const Model<T, MODE>& m, const T* p, bool circular,
                             T (&alpha)[Np<MODE>::v][Np<MODE>::v], T (&beta)[Np<MODE>::v])
{
	constexpr int NP = Np<MODE>::v;
	const int lane = threadIdx.x & 31;
	T err = T(0);
	#pragma unroll
	for (int a = 0; a < NP; ++a) {
		beta[a] = T(0);
		#pragma unroll
		for (int b = a; b < NP; ++b) { alpha[a][b] = T(0); }
	}
	int i = lane / R.roi, j = lane - i * R.roi;
	for (int idx = lane; idx < R.n; idx += 32) {
		const T v = static_cast<T>(__ldg(R.base + static_cast<long long>(i) * R.W + j));
		T g[NP];
		const T hat = m.template Eval<true>(R.x0 + T(j) - p[2], R.x0 + T(i) - p[3], g);
		if constexpr (MODE == kG3Theta) {
			if (circular) { g[6] = T(0); }
		}
		const T d = v - hat;
		err += d * d;
		#pragma unroll
		for (int a = 0; a < NP; ++a) {
			beta[a] += g[a] * d;
			#pragma unroll
			for (int b = a; b < NP; ++b) { alpha[a][b] += g[a] * g[b]; }
		}
		j += 32;
		while (j >= R.roi) { j -= R.roi; ++i; }
	}
	err = WarpSum(err);
	#pragma unroll
	for (int a = 0; a < NP; ++a) {
		beta[a] = WarpSum(beta[a]);
		#pragma unroll
		for (int b = a; b < NP; ++b) {
			alpha[a][b] = WarpSum(alpha[a][b]);
			alpha[b][a] = alpha[a][b];
		}
	}
	return err;
}

template <typename T, int MODE>
__device__ T TrialError(const Roi<T, MODE>& R, const Model<T, MODE>& m, const T* p)
{
	const int lane = threadIdx.x & 31;
	T res = T(0);
	int i = lane / R.roi, j = lane - i * R.roi;
	for (int idx = lane; idx < R.n; idx += 32) {
		const T v = static_cast<T>(__ldg(R.base + static_cast<long long>(i) * R.W + j));
		const T d = v - m.template Eval<false>(R.x0 + T(j) - p[2], R.x0 + T(i) - p[3], nullptr);
		res += d * d;
		j += 32;
		while (j >= R.roi) { j -= R.roi; ++i; }
	}
	return WarpSum(res);
}

// Squared correlation between data and model (GaussianFit.cpp:274-295).
template <typename T, int MODE>
__device__ double SquaredCorrelation(const Roi<T, MODE>& R, const Model<T, MODE>& m, const T* p)
{
	const int lane = threadIdx.x & 31;
	double sd = 0, sm = 0;
	int i = lane / R.roi, j = lane - i * R.roi;
	for (int idx = lane; idx < R.n; idx += 32) {
		sd += static_cast<double>(__ldg(R.base + static_cast<long long>(i) * R.W + j));
		sm += static_cast<double>(m.template Eval<false>(R.x0 + T(j) - p[2], R.x0 + T(i) - p[3], nullptr));
		j += 32;
		while (j >= R.roi) { j -= R.roi; ++i; }
	}
	const double muD = WarpSum(sd) / R.n, muM = WarpSum(sm) / R.n;
	double t1 = 0, t2 = 0, t3 = 0;
	i = lane / R.roi;
	j = lane - i * R.roi;
	for (int idx = lane; idx < R.n; idx += 32) {
		const double d = static_cast<double>(__ldg(R.base + static_cast<long long>(i) * R.W + j)) - muD;
		const double h = static_cast<double>(m.template Eval<false>(R.x0 + T(j) - p[2], R.x0 + T(i) - p[3], nullptr)) - muM;
		t1 += d * h;
		t2 += d * d;
		t3 += h * h;
		j += 32;
		while (j >= R.roi) { j -= R.roi; ++i; }
	}
	t1 = WarpSum(t1);
	t2 = WarpSum(t2);
	t3 = WarpSum(t3);
	const double r = t1 / sqrt(t2 * t3);
	return isnan(r) ? 0.0 : r * r;
}

// Returns 0 = fitted row stored, 1 = sentinel row stored. `converged` reports a clean stop (FP32 screening).
template <typename T, int MODE>
__device__ void FitOne(const uint16_t* frame, int H, int W, const FitParams& fp, const Cand& cd, double* row,
                       bool* cleanOut)
{
	constexpr int NP = Np<MODE>::v;
	const int half = fp.half;
	bool clean = true;
	// border test on the truncated centroid (GaussianFit.cpp:51-56), unsigned as in the reference
	const bool nonneg = cd.x >= 0.0 && cd.y >= 0.0;  // negative or NaN positions fail the reference test too
	const unsigned long long ux = nonneg ? static_cast<unsigned long long>(cd.x) : 0ull;
	const unsigned long long uy = nonneg ? static_cast<unsigned long long>(cd.y) : 0ull;
	const unsigned long long h = static_cast<unsigned long long>(half);
	if (!nonneg || h > ux || ux >= static_cast<unsigned long long>(W) - h || h > uy || uy >= static_cast<unsigned long long>(H) - h) {
		StoreRow(row, MODE, cd.intensity, cd.surf, cd.x, cd.y, 0, -1, -1, -1, -1, -1, -1, -1);
		if (cleanOut) { *cleanOut = true; }
		return;
	}
	Roi<T, MODE> R;
	R.base = frame + static_cast<long long>(uy - h) * W + static_cast<long long>(ux - h);
	R.W = W;
	R.roi = fp.roi;
	R.n = fp.n;
	R.x0 = T(-half);
	// ROI min / max (Fitting.cpp:109-123)
	const int lane = threadIdx.x & 31;
	T vmin = T(1e30), vmax = T(-1e30);
	{
		int i = lane / R.roi, j = lane - i * R.roi;
		for (int idx = lane; idx < R.n; idx += 32) {
			const T v = static_cast<T>(__ldg(R.base + static_cast<long long>(i) * W + j));
			vmin = min(vmin, v);
			vmax = max(vmax, v);
			j += 32;
			while (j >= R.roi) { j -= R.roi; ++i; }
		}
		vmin = WarpMin(vmin);
		vmax = WarpMax(vmax);
	}
	// initial parameters and bounds in local coordinates (Fitting.cpp:126-175)
	const T lx = static_cast<T>(cd.x - static_cast<double>(ux)), ly = static_cast<T>(cd.y - static_cast<double>(uy));
	T p[NP], lo[NP], hi[NP];
	p[0] = vmin; p[1] = vmax - vmin; p[2] = lx; p[3] = ly;
	lo[0] = T(0); lo[1] = T(0); lo[2] = lx - T(1); lo[3] = ly - T(1);
	hi[0] = T(65535); hi[1] = T(65535); hi[2] = lx + T(1); hi[3] = ly + T(1);
	const T sqrt2 = T(1.4142135623730951);
	if constexpr (MODE == kG2Sigma) { p[4] = T(fp.sigmaX); lo[4] = T(0.1); hi[4] = T(20); }
	if constexpr (MODE == kG3Fixed || MODE == kG3Theta) {
		p[4] = sqrt2 * T(fp.sigmaX); p[5] = sqrt2 * T(fp.sigmaY);
		lo[4] = lo[5] = T(0.1);
		hi[4] = hi[5] = T(20);
	}
	if constexpr (MODE == kG3Theta) { p[6] = T(fp.theta); lo[6] = T(-150); hi[6] = T(150); }
	const T sigma0 = T(fp.sigmaX), theta0 = T(fp.theta);
	const T dblEps = T(2.220446049250313e-16);

	T alpha[NP][NP], beta[NP], dp[NP], pTry[NP];
	Model<T, MODE> model;
	auto normal = [&]() {
		model.Make(p, sigma0, theta0);
		const bool circular = MODE == kG3Theta && fabs(p[4] - p[5]) <= dblEps;
		return NormalEquations<T, MODE>(R, model, p, circular, alpha, beta);
	};
	auto maxAbsBeta = [&]() {
		T m = T(0);
		#pragma unroll
		for (int a = 0; a < NP; ++a) { m = max(m, fabs(beta[a])); }
		return m;
	};
	auto relStep = [&]() {
		T m = T(0);
		#pragma unroll
		for (int a = 0; a < NP; ++a) { m = max(m, fabs(dp[a]) / max(fabs(p[a]), T(1e-12))); }
		return m;
	};
	auto fail = [&]() { StoreRow(row, MODE, cd.intensity, cd.surf, cd.x, cd.y, 0, -1, -1, -1, -1, -1, -1, -1); };

	T err = normal();
	bool finite = Finite(err);
	#pragma unroll
	for (int a = 0; a < NP; ++a) { finite = finite && Finite(beta[a]); }
	if (!finite) { fail(); if (cleanOut) { *cleanOut = true; } return; }
	T lambda = T(1e-2);
	const T lamMax = T(1e7), lamMin = T(1e-7);
	T m = maxAbsBeta();
	int it = (m < T(1e-6)) ? kMaxIter : 0;
	for (; it < kMaxIter; ++it) {
		if (!Solve<T, NP>(alpha, beta, lambda, dp)) {
			if (lambda < lamMax) { lambda = min(lambda * T(11), lamMax); continue; }
			fail();
			if (cleanOut) { *cleanOut = sizeof(T) == 8; }
			return;
		}
		bool dpFinite = true;
		#pragma unroll
		for (int a = 0; a < NP; ++a) {
			dpFinite = dpFinite && Finite(dp[a]);
			pTry[a] = min(max(p[a] + dp[a], lo[a]), hi[a]);
		}
		if (!dpFinite) { fail(); if (cleanOut) { *cleanOut = sizeof(T) == 8; } return; }
		bool tiny = true;
		#pragma unroll
		for (int a = 0; a < NP; ++a) {
			dp[a] = pTry[a] - p[a];
			tiny = tiny && fabs(dp[a]) < T(1e-15);
		}
		if (tiny) {
			if (lambda >= lamMax) { break; }
			lambda = min(lambda * T(11), lamMax);
			continue;
		}
		// predicted gain 2 dp.beta - dp.alpha.dp (GaussianFit.cpp:248-259)
		T quad = T(0), lin = T(0);
		#pragma unroll
		for (int a = 0; a < NP; ++a) {
			T t = T(0);
			#pragma unroll
			for (int b = 0; b < NP; ++b) { t += alpha[a][b] * dp[b]; }
			quad += dp[a] * t;
			lin += dp[a] * beta[a];
		}
		const T gain = (T(2) * lin) - quad;
		if (gain <= T(0)) {
			if (lambda >= lamMax) { break; }
			lambda = min(lambda * T(11), lamMax);
			if (relStep() < T(1e-6) && it >= 2) { break; }
			continue;
		}
		T denom = T(0);
		#pragma unroll
		for (int a = 0; a < NP; ++a) { denom += dp[a] * ((lambda * dp[a]) + beta[a]); }
		Model<T, MODE> trial;
		trial.Make(pTry, sigma0, theta0);
		const T errTry = TrialError<T, MODE>(R, trial, pTry);
		const T rho = (err - errTry) / (T(2) * denom);
		if (rho > T(1e-2)) {
			#pragma unroll
			for (int a = 0; a < NP; ++a) { p[a] = pTry[a]; }
			err = normal();
			lambda = max(lambda / T(9), lamMin);
		}
		else {
			if (lambda >= lamMax) { break; }
			lambda = min(lambda * T(11), lamMax);
		}
		if (it >= 2) {
			if (relStep() < T(1e-6)) { break; }
			if (err / T(R.n) < T(1e-5)) { break; }
			if (maxAbsBeta() < T(1e-6)) { break; }
		}
	}
	if (it >= kMaxIter) { clean = false; }  // ran out of iterations: an FP32 result is re-done in FP64
	model.Make(p, sigma0, theta0);
	const double r2 = SquaredCorrelation<T, MODE>(R, model, p);
	const double x = static_cast<double>(ux) + static_cast<double>(p[2]);
	const double y = static_cast<double>(uy) + static_cast<double>(p[3]);
	if (cleanOut) { *cleanOut = clean; }
	if (r2 < kEps) {
		StoreRow(row, MODE, cd.intensity, cd.surf, x, y, 0, -1, -1, -1, -1, -1, -1, -1);
		return;
	}
	double sx = fp.sigmaX, sy = fp.sigmaY, th = fp.theta;
	if constexpr (MODE == kG2Fixed) { sx = sy = fp.sigmaX; th = 0; }
	if constexpr (MODE == kG2Sigma) { sx = static_cast<double>(p[4]); sy = sx; th = 0; }
	if constexpr (MODE == kG3Fixed || MODE == kG3Theta) {
		sx = static_cast<double>(p[4]) / 1.4142135623730951;
		sy = static_cast<double>(p[5]) / 1.4142135623730951;
	}
	if constexpr (MODE == kG3Theta) { th = static_cast<double>(p[6]); }
	StoreRow(row, MODE, cd.intensity, cd.surf, x, y, 0, static_cast<double>(p[0]), static_cast<double>(p[1]), sx, sy, th, r2, -1);
}

// One warp per candidate. FP32 instances flag candidates that must be re-fitted in FP64.
template <typename T, int MODE>
__global__ void __launch_bounds__(128) GaussFitKernel(const uint16_t* __restrict__ img, int H, int W, long long N,
                                                      const Cand* __restrict__ cands, const uint32_t* nptr, uint32_t nconst,
                                                      FitParams fp, double* rows, uint8_t* flags, const uint8_t* only)
{
	const uint32_t n = nptr ? *nptr : nconst;
	const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
	for (uint32_t k = warp; k < n; k += nw) {
		if (only && !only[k]) { continue; }
		const Cand cd = cands[k];
		bool clean = true;
		FitOne<T, MODE>(img + static_cast<long long>(cd.frame) * N, H, W, fp, cd, rows + static_cast<long long>(k) * kCols,
		                flags ? &clean : nullptr);
		if (flags && (threadIdx.x & 31) == 0) { flags[k] = clean ? 0 : 1; }
	}
}

// Mode 0 (and any mode without a model): the segmentation values only (Fitting.hpp:63-66).
__global__ void NoFitKernel(const Cand* __restrict__ cands, const uint32_t* nptr, uint32_t nconst, double* rows)
{
	const uint32_t n = nptr ? *nptr : nconst;
	for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
		const Cand cd = cands[k];
		double* r = rows + static_cast<long long>(k) * kCols;
		r[cId] = 0; r[cPlane] = 0; r[cIndex] = 0; r[cChannel] = -1;
		r[cX] = cd.x; r[cY] = cd.y; r[cZ] = 0;
		r[cIntensity] = cd.intensity;
		r[cSigmaX] = -1; r[cSigmaY] = -1; r[cTheta] = -1; r[cQualityXY] = -1; r[cQualityZ] = -1;
		r[cAmplitude] = 0; r[cOffset] = 0;
		r[cSegIntensity] = cd.intensity; r[cSurface] = cd.surf;
		r[cCircularity] = 1;
	}
}

template <typename T>
bool LaunchGaussT(const uint16_t* img, int H, int W, long long N, const Cand* cands, const uint32_t* nptr, uint32_t nconst,
                  uint32_t cap, const FitParams& fp, double* rows, uint8_t* flags, const uint8_t* only, cudaStream_t st)
{
	const int threads = 128;
	const uint32_t warps = cap > 0 ? cap : 1;
	const uint32_t blocks = std::min<uint32_t>((warps + 3) / 4, 148u * 16u);
	switch (fp.mode) {
		case kG2Fixed: GaussFitKernel<T, kG2Fixed><<<blocks, threads, 0, st>>>(img, H, W, N, cands, nptr, nconst, fp, rows, flags, only); break;
		case kG2Sigma: GaussFitKernel<T, kG2Sigma><<<blocks, threads, 0, st>>>(img, H, W, N, cands, nptr, nconst, fp, rows, flags, only); break;
		case kG3Fixed: GaussFitKernel<T, kG3Fixed><<<blocks, threads, 0, st>>>(img, H, W, N, cands, nptr, nconst, fp, rows, flags, only); break;
		case kG3Theta: GaussFitKernel<T, kG3Theta><<<blocks, threads, 0, st>>>(img, H, W, N, cands, nptr, nconst, fp, rows, flags, only); break;
		default: return false;
	}
	CountLaunch();
	return PTB_LAUNCHED();
}

}  // namespace

bool LaunchSpline(const uint16_t* img, int H, int W, long long N, const Cand* cands, const uint32_t* nptr, uint32_t nconst,
                  uint32_t cap, const FitParams& fp, double* rows, cudaStream_t st);
bool LaunchMle(int lanes, const FitImages& fi, const Cand* cands, const uint32_t* nptr, uint32_t nconst,
               uint32_t cap, const MleParams& mp, double* rows, cudaEvent_t* marks, cudaStream_t st);
bool LaunchExactFit(const uint16_t* img, int H, int W, long long N, const Cand* cands, const uint32_t* nptr, uint32_t nconst,
                    uint32_t cap, const FitParams& fp, double* rows, const uint8_t* only, cudaStream_t st);

// Fits `n` candidates (device count *nptr, or nconst when nptr is null; `cap` bounds it) into rows[k * 18].
// precision 0: FP64 in the reference's order (thread per ROI); 1: FP32 warp-per-ROI first, then the FP64 exact
// kernel for the candidates the FP32 pass flags; 2: FP64 warp-per-ROI.
bool LaunchFit(const uint16_t* img, int H, int W, long long N, const Cand* cands, const uint32_t* nptr, uint32_t nconst,
               uint32_t cap, const FitParams& fp, double* rows, uint8_t* flags, int precision, cudaStream_t st)
{
	if (fp.mode == kSplineEmccd) { return LaunchSpline(img, H, W, N, cands, nptr, nconst, cap, fp, rows, st); }
	if (fp.mode >= kMleGauss && fp.mode <= kMleSpline) {
		return LaunchMle(fp.lanes, OneImage(img, H, W, N), cands, nptr, nconst, cap, fp.mle, rows, fp.marks, st);
	}
	if (fp.mode < kG2Fixed || fp.mode > kG3Theta) {
		const uint32_t blocks = std::min<uint32_t>((cap + 255) / 256 + 1, 148u * 8u);
		NoFitKernel<<<blocks, 256, 0, st>>>(cands, nptr, nconst, rows);
		CountLaunch();
		return PTB_LAUNCHED();
	}
	if (precision == 1 && flags) {
		bool ok = LaunchGaussT<float>(img, H, W, N, cands, nptr, nconst, cap, fp, rows, flags, nullptr, st);
		return ok && LaunchExactFit(img, H, W, N, cands, nptr, nconst, cap, fp, rows, flags, st);
	}
	if (precision == 2) { return LaunchGaussT<double>(img, H, W, N, cands, nptr, nconst, cap, fp, rows, nullptr, nullptr, st); }
	return LaunchExactFit(img, H, W, N, cands, nptr, nconst, cap, fp, rows, nullptr, st);
}

}  // namespace ptb
