// Poisson maximum-likelihood fits (modes 6 Gaussian, 7 astigmatic 3D, 8 cubic-spline 3D) of (bg, I, x, y, s),
// s = sigma (mode 6), z in nm (mode 7) or the spline's z coordinate (mode 8). No counterpart in the reference; the
// model maths and the FP64 oracle are in oracle/pt_oracle.cpp (MleFit). This file follows it: the same initial
// values, bounds and axial pre-scan (here in FP32), the same damped Fisher-scoring LM on the Poisson deviance (its
// step-size stop rule two decades looser, see StepSmall), then Newton steps on the exact Hessian of the deviance,
// parameters on active bounds held throughout, and the CRLB from the Fisher information at the final point.
//
// Precision: the LM iterations and the Newton polish run in FP32, with the hardware approximations of exp and log
// (__expf: a few ulp; __logf: absolute error about 2^-21 near 1) and erff; the per-pixel logarithm of the deviance
// had been a fifth of the LM's time. Each 5x5 system is factored by an FP32 Cholesky;
// when a pivot is not positive or the pivot ratio min(L_ii^2 / A_ii) falls below 1e-5 the same system is
// re-factored in FP64. The final pass forms the deviance (reported in the Theta column) and the Fisher information
// behind the CRLB in FP64; the initial axial pre-scan, a handful of deviance
// evaluations that choose the starting basin, runs in FP32 like the LM. The oracle
// polishes in FP64 to a 1e-10 relative step; the FP32 polish stops at a 1e-6 relative step (the FP32 resolution of
// the deviance), well inside the stated tolerance of 1e-3 px and 1e-4 relative photons.
//
// Two mappings, chosen per (mode, ROI) by the autotuner in engine.cu:
//   * thread per ROI, four launches that hand their state over in the output rows (columns 0-4 theta, column 5 a
//     status) so that no extra device memory is needed:
//       MleInitKernel   initial values and axial pre-scan;
//       MleLmKernel     persistent FP32 LM: every warp owns a contiguous range of candidates and each lane takes the
//                       next candidate of the range as soon as its own converges, so a lane never idles while the
//                       other 31 iterate; ROI photons and the column erf factors are staged per lane in shared memory;
//       MlePolishKernel persistent FP32 Newton polish, organised the same way;
//       MleFinalKernel  FP64 Fisher information, CRLB, output row;
//   * warp per ROI (MleWarpKernel): all four phases in one launch, pixels spread over the lanes, sums reduced with
//     shuffles; better for large ROIs and for the spline model, whose 64 coefficients per pixel dominate.
// For modes 6-7 the pixel-integrated Gaussian is separable: the erf factors are formed once per ROI column and row
// per evaluation. The spline table is cell-major ([cell][64]) in FP32 for the FP32 phases and in FP64 for the FP64
// ones.
#include <algorithm>
#include <mutex>
#include <type_traits>

#include "pt_common.cuh"

namespace ptb {

namespace {

constexpr int kMaxRoi = 15;
constexpr int kMaxPix = kMaxRoi * kMaxRoi;
constexpr int kThreads = 64;

// State handed between the thread-per-ROI launches in column kStatusCol of the output row.
constexpr int kStatusCol = 5;
constexpr double kStOk = 0.0, kStFailed = 1.0, kStBorder = 2.0;

// What one evaluation accumulates: deviance only; deviance, gradient and Fisher-scoring matrix; deviance, gradient,
// exact Hessian and Fisher information; deviance and Fisher information (the FP64 final pass: the log-likelihood and
// CRLB of the result).
enum Kind { kDevOnly = 0, kFisher = 1, kExact = 2, kFinal = 3 };

template <int KIND> struct Fields { static constexpr int value = KIND == kDevOnly ? 1 : (KIND == kExact ? 6 : 3); };

template <typename T> __device__ __forceinline__ T Erf(T x);
template <> __device__ __forceinline__ float Erf<float>(float x) { return erff(x); }
template <> __device__ __forceinline__ double Erf<double>(double x) { return erf(x); }
template <typename T> __device__ __forceinline__ T Ex(T x);
template <> __device__ __forceinline__ float Ex<float>(float x) { return __expf(x); }  // hardware ex2 based
template <> __device__ __forceinline__ double Ex<double>(double x) { return exp(x); }
template <typename T> __device__ __forceinline__ T Ln(T x);
template <> __device__ __forceinline__ float Ln<float>(float x) { return __logf(x); }  // hardware lg2 based
template <> __device__ __forceinline__ double Ln<double>(double x) { return log(x); }

// Division in the per-pixel sums: FP32 with the hardware approximation (divisors here are photon counts and model
// values, far inside its range), FP64 exact.
template <typename T> __device__ __forceinline__ T Div(T a, T b) { return a / b; }
template <> __device__ __forceinline__ float Div<float>(float a, float b) { return __fdividef(a, b); }

// Lanes of the calling lane's group of L consecutive lanes (L a power of two, the groups of a warp disjoint).
template <int L>
__device__ __forceinline__ unsigned GroupMask()
{
	if constexpr (L >= 32) { return 0xffffffffu; }
	else { return ((1u << L) - 1u) << ((threadIdx.x & 31) & ~(L - 1)); }
}

// Sum over the calling lane's group of L lanes; every lane of the group receives the same value (each butterfly step
// adds the same two partial sums on both partners, and addition is commutative).
template <int L, typename T>
__device__ __forceinline__ T GroupSum(T v)
{
	#pragma unroll
	for (int d = L / 2; d > 0; d >>= 1) { v += __shfl_xor_sync(GroupMask<L>(), v, d); }
	return v;
}

// Pixel-integrated 1D Gaussian factor E = (erf(b) - erf(a)) / 2, a = (c - x - 1/2) k, b = (c - x + 1/2) k,
// k = 1 / (sqrt2 s), and its derivatives in the position and the width (NF >= 3) and the second derivatives E_xx,
// E_xs, E_ss (NF == 6).
template <typename T>
struct Fac {
	T e, dx, ds, xx, xs, ss;
};

// The factors are formed from values at the pixel boundaries: pixel j spans boundaries j and j + 1, so a row of roi pixels
// needs roi + 1 erf and exp evaluations instead of 2 roi. Boundary u at z = ((u - h) - x - 1/2) k, k = 1 / (sqrt2 s):
// E = erf(z), Q0 = exp(-z^2), Q1 = z Q0, Q2 = z Q1, Q3 = z Q2; with r1 = 1 / (sqrt(2 pi) s), r2 = 1 / (sqrt(pi) s)
// the factor of pixel [a, b] is e = (E_b - E_a) / 2, dx = (Q0_a - Q0_b) r1, ds = (Q1_a - Q1_b) r2 and
// xx = ds / s, xs = (2 (Q2_a - Q2_b) - Q0_a + Q0_b) r1 / s, ss = 2 (Q3_a - Q1_a - Q3_b + Q1_b) r2 / s.
template <typename T>
struct Bound {
	T E, Q0, Q1, Q2, Q3;
};

template <typename T>
struct AxisConst {
	T k, r1, r2, inv;
	__device__ __forceinline__ explicit AxisConst(T s)
	{
		k = T(1) / (T(1.4142135623730951) * s);
		r1 = T(1) / (T(2.5066282746310002) * s);
		r2 = T(1) / (T(1.7724538509055160) * s);
		inv = T(1) / s;
	}
};

template <typename T, int NF>
__device__ __forceinline__ Bound<T> MakeBound(int u, int h, T x, T k)
{
	Bound<T> b;
	const T z = (T(u - h) - x - T(0.5)) * k;
	b.E = Erf<T>(z);
	b.Q0 = b.Q1 = b.Q2 = b.Q3 = T(0);
	if constexpr (NF >= 3) {
		b.Q0 = Ex<T>(-z * z);
		b.Q1 = z * b.Q0;
		if constexpr (NF == 6) {
			b.Q2 = z * b.Q1;
			b.Q3 = z * b.Q2;
		}
	}
	return b;
}

template <typename T, int NF>
__device__ __forceinline__ Fac<T> FacOf(const Bound<T>& a, const Bound<T>& b, const AxisConst<T>& ac)
{
	Fac<T> f;
	f.e = T(0.5) * (b.E - a.E);
	f.dx = f.ds = f.xx = f.xs = f.ss = T(0);
	if constexpr (NF >= 3) {
		f.dx = (a.Q0 - b.Q0) * ac.r1;
		f.ds = (a.Q1 - b.Q1) * ac.r2;
		if constexpr (NF == 6) {
			f.xx = f.ds * ac.inv;
			f.xs = (T(2) * (a.Q2 - b.Q2) - a.Q0 + b.Q0) * ac.r1 * ac.inv;
			f.ss = T(2) * (a.Q3 - a.Q1 - b.Q3 + b.Q1) * ac.r2 * ac.inv;
		}
	}
	return f;
}

// Factor table in shared memory: field f of entry c at p[(c * NF + f) * s].
template <typename T>
struct FacTab {
	T* p;
	int s;
	template <int NF>
	__device__ __forceinline__ void Put(int c, const Fac<T>& f) const
	{
		T* q = p + c * NF * s;
		q[0] = f.e;
		if constexpr (NF >= 3) { q[s] = f.dx; q[2 * s] = f.ds; }
		if constexpr (NF == 6) { q[3 * s] = f.xx; q[4 * s] = f.xs; q[5 * s] = f.ss; }
	}
	template <int NF>
	__device__ __forceinline__ Fac<T> Get(int c) const
	{
		const T* q = p + c * NF * s;
		Fac<T> f;
		f.e = q[0];
		f.dx = f.ds = f.xx = f.xs = f.ss = T(0);
		if constexpr (NF >= 3) { f.dx = q[s]; f.ds = q[2 * s]; }
		if constexpr (NF == 6) { f.xx = q[3 * s]; f.xs = q[4 * s]; f.ss = q[5 * s]; }
		return f;
	}
};

// Astigmatic width (pixels) and its first and second z derivatives for one axis [z0, w, c3, c4, A].
template <typename T>
__device__ __forceinline__ void AstigSigma(const double* m, double pixelSize, T z, T& s, T& ds, T& dss)
{
	const T u = (z - T(m[0])) / T(m[1]);
	const T poly = T(1) + u * u + T(m[2]) * u * u * u + T(m[3]) * u * u * u * u;
	const T k = T(m[4] / pixelSize);
	if (poly <= T(1e-12)) { s = k * T(1e-6); ds = T(0); dss = T(0); return; }
	const T r = sqrt(poly);
	const T p1 = T(2) * u + T(3 * m[2]) * u * u + T(4 * m[3]) * u * u * u;
	const T p2 = T(2) + T(6 * m[2]) * u + T(12 * m[3]) * u * u;
	s = k * r;
	ds = k * p1 / (T(2) * r * T(m[1]));
	dss = k / (T(m[1]) * T(m[1])) * (p2 / (T(2) * r) - p1 * p1 / (T(4) * r * poly));
}

// Separable PSF at one pixel; P1 = d psf / d(x, y, s), P2 = the second derivatives (xx, xy, xs, yy, ys, ss).
template <typename T, int NF>
__device__ __forceinline__ T GaussPixel(const Fac<T>& X, const Fac<T>& Y, T dsx, T dsy, T ssx, T ssy, T P1[3], T P2[6])
{
	if constexpr (NF >= 3) {
		P1[0] = X.dx * Y.e;
		P1[1] = X.e * Y.dx;
		P1[2] = X.ds * dsx * Y.e + X.e * Y.ds * dsy;
	}
	if constexpr (NF == 6) {
		P2[0] = X.xx * Y.e;
		P2[1] = X.dx * Y.dx;
		P2[2] = X.xs * dsx * Y.e + X.dx * Y.ds * dsy;
		P2[3] = X.e * Y.xx;
		P2[4] = X.ds * dsx * Y.dx + X.e * Y.xs * dsy;
		P2[5] = (X.ss * dsx * dsx + X.ds * ssx) * Y.e + T(2) * X.ds * dsx * Y.ds * dsy + X.e * (Y.ss * dsy * dsy + Y.ds * ssy);
	}
	return X.e * Y.e;
}

__device__ __forceinline__ int SplineCell(double v, int dim) { return min(max(static_cast<int>(floor(v)), 0), dim - 1); }
__device__ __forceinline__ int SplineCell(float v, int dim) { return min(max(static_cast<int>(floorf(v)), 0), dim - 1); }

// Cubic-spline PSF at table coordinates (X, Y, Z): the cell index is clamped to the table and the fraction taken
// from the clamped cell, as in the oracle. P1 and P2 are the derivatives in the fit parameters (x, y, s): X and Y
// decrease as x and y grow, so their odd derivatives change sign.
template <typename T, int NF>
__device__ __forceinline__ T SplinePixel(const MleParams& mp, T X, T Y, T Z, T P1[3], T P2[6])
{
	const int ix = SplineCell(X, mp.sx), iy = SplineCell(Y, mp.sy), iz = SplineCell(Z, mp.sz);
	const T f[3] = {X - T(ix), Y - T(iy), Z - T(iz)};
	T p[3][4], d[3][4], dd[3][4];
	#pragma unroll
	for (int a = 0; a < 3; ++a) {
		p[a][0] = T(1); p[a][1] = f[a]; p[a][2] = f[a] * f[a]; p[a][3] = f[a] * f[a] * f[a];
		d[a][0] = T(0); d[a][1] = T(1); d[a][2] = T(2) * f[a]; d[a][3] = T(3) * f[a] * f[a];
		dd[a][0] = T(0); dd[a][1] = T(0); dd[a][2] = T(2); dd[a][3] = T(6) * f[a];
	}
	const long long cell = (static_cast<long long>(iz) * mp.sy + iy) * mp.sx + ix;
	T v = T(0), sX = T(0), sY = T(0), sZ = T(0), sXX = T(0), sXY = T(0), sXZ = T(0), sYY = T(0), sYZ = T(0), sZZ = T(0);
	#pragma unroll
	for (int q = 0; q < 16; ++q) {  // q = zi * 4 + yj: the four x-monomials of one (z, y) pair
		T c0, c1, c2, c3;
		if constexpr (std::is_same<T, float>::value) {
			const float4 c = __ldg(reinterpret_cast<const float4*>(mp.table + cell * 64) + q);
			c0 = c.x; c1 = c.y; c2 = c.z; c3 = c.w;
		}
		else {
			const double2 a = __ldg(reinterpret_cast<const double2*>(mp.table64 + cell * 64) + 2 * q);
			const double2 b = __ldg(reinterpret_cast<const double2*>(mp.table64 + cell * 64) + 2 * q + 1);
			c0 = a.x; c1 = a.y; c2 = b.x; c3 = b.y;
		}
		const int zi = q >> 2, yj = q & 3;
		const T sx = c0 * p[0][0] + c1 * p[0][1] + c2 * p[0][2] + c3 * p[0][3];
		const T zy = p[2][zi] * p[1][yj];
		v += zy * sx;
		if constexpr (NF >= 3) {
			const T dx = c1 * d[0][1] + c2 * d[0][2] + c3 * d[0][3];
			sX += zy * dx;
			sY += p[2][zi] * d[1][yj] * sx;
			sZ += d[2][zi] * p[1][yj] * sx;
			if constexpr (NF == 6) {
				const T ddx = c2 * dd[0][2] + c3 * dd[0][3];
				sXX += zy * ddx;
				sXY += p[2][zi] * d[1][yj] * dx;
				sXZ += d[2][zi] * p[1][yj] * dx;
				sYY += p[2][zi] * dd[1][yj] * sx;
				sYZ += d[2][zi] * d[1][yj] * sx;
				sZZ += dd[2][zi] * p[1][yj] * sx;
			}
		}
	}
	if constexpr (NF >= 3) { P1[0] = -sX; P1[1] = -sY; P1[2] = sZ; }
	if constexpr (NF == 6) { P2[0] = sXX; P2[1] = sXY; P2[2] = -sXZ; P2[3] = sYY; P2[4] = -sYZ; P2[5] = sZZ; }
	return v;
}

// One pixel's share of the sums. Fisher scoring: Hm = 2 sum dmu dmu^T / mu. Exact: Hm = the Hessian of the deviance,
// 2 sum [d / mu^2 dmu dmu^T + (1 - d / mu) d2mu], and Fm = sum dmu dmu^T / mu (Fisher information). Final: Fm only.
template <typename T, int KIND>
__device__ __forceinline__ void Accumulate(T d, T bg, T I, T psf, const T P1[3], const T P2[6], T& D, T G[5], T Hm[15], T Fm[15])
{
	const T mu = max(bg + I * psf, T(1e-6));
	if constexpr (KIND == kFinal) {
		// FP64: log(mu / d) = -log(d * (1 / mu)), the reciprocal shared with the Fisher weights (one FP64 division
		// per pixel instead of two; the two forms differ by an ulp of the ratio)
		const T rmu = T(1) / mu;
		D += d > T(0) ? T(2) * (mu - d + d * Ln<T>(d * rmu)) : T(2) * mu;
		const T gk[5] = {T(1), psf, I * P1[0], I * P1[1], I * P1[2]};
		int q = 0;
		#pragma unroll
		for (int a = 0; a < 5; ++a) {
			const T wa = rmu * gk[a];
			#pragma unroll
			for (int b = a; b < 5; ++b) { Fm[q++] += wa * gk[b]; }
		}
		return;
	}
	D += d > T(0) ? T(2) * (mu - d - d * Ln<T>(Div<T>(mu, d))) : T(2) * mu;
	if constexpr (KIND != kDevOnly) {
		const T gk[5] = {T(1), psf, I * P1[0], I * P1[1], I * P1[2]};
		const T rmu = Div<T>(T(1), mu);
		const T w1 = T(2) * (T(1) - d * rmu);
		const T w2 = KIND == kExact ? T(2) * d * rmu * rmu : T(2) * rmu;
		int q = 0;
		#pragma unroll
		for (int a = 0; a < 5; ++a) {
			G[a] += w1 * gk[a];
			const T wa = w2 * gk[a];
			#pragma unroll
			for (int b = a; b < 5; ++b) { Hm[q++] += wa * gk[b]; }
		}
		if constexpr (KIND == kExact) {
			// d2mu in the packed upper triangle: (I, x) = Px, (I, y) = Py, (I, s) = Ps, (x, x) = I Pxx, ...
			Hm[6] += w1 * P1[0];
			Hm[7] += w1 * P1[1];
			Hm[8] += w1 * P1[2];
			Hm[9] += w1 * I * P2[0];
			Hm[10] += w1 * I * P2[1];
			Hm[11] += w1 * I * P2[2];
			Hm[12] += w1 * I * P2[3];
			Hm[13] += w1 * I * P2[4];
			Hm[14] += w1 * I * P2[5];
		}
	}
}

// Where an evaluation reads the ROI's photons: FP32 photons staged in shared memory (pixel k at sm[k * ss]), or the
// frame (FP64 evaluations, and FP32 ones without staging).
struct Pix {
	const float* sm;
	int ss;
	const uint16_t* g;  // ROI origin in the frame
	int W;
	float off32, inv32;
	double off64, inv64;
};

template <typename T>
__device__ __forceinline__ T Photons(const Pix& px, int i, int j, int k)
{
	if constexpr (std::is_same<T, float>::value) {
		if (px.sm) { return px.sm[k * px.ss]; }
		return fmaxf((float(__ldg(px.g + i * px.W + j)) - px.off32) * px.inv32, 0.f);
	}
	else { return fmax((double(__ldg(px.g + i * px.W + j)) - px.off64) * px.inv64, 0.0); }
}

// Deviance D at theta and, by KIND, the gradient G, the curvature Hm and the Fisher information Fm (upper
// triangles, 15 entries). L = 1: the calling thread sums the whole ROI, the column factors go to its table xt. L > 1:
// a group of L consecutive lanes (the warp for L = 32) shares the pixels, the column and row factors go to the group's
// tables xt and yt, the sums are reduced over the group and every lane of it returns them. All lanes of a group call
// it together.
template <typename T, int MODEL, int L, int KIND>
__device__ T Normal(const MleParams& mp, const Pix& px, const T th[5], T G[5], T Hm[15], T Fm[15], FacTab<T> xt, FacTab<T> yt)
{
	constexpr int NF = Fields<KIND>::value;
	const int roi = mp.roi, h = mp.half, n = mp.n;
	const int gl = L == 1 ? 0 : static_cast<int>(threadIdx.x & (L - 1));
	T sx = th[4], sy = th[4], dsx = T(1), dsy = T(1), ssx = T(0), ssy = T(0);
	if constexpr (MODEL == 7) {
		AstigSigma<T>(mp.astig, mp.pixelSize, th[4], sx, dsx, ssx);
		AstigSigma<T>(mp.astig + 5, mp.pixelSize, th[4], sy, dsy, ssy);
	}
	T D = T(0);
	if constexpr (KIND == kFisher || KIND == kExact) {
		#pragma unroll
		for (int a = 0; a < 5; ++a) { G[a] = T(0); }
		#pragma unroll
		for (int a = 0; a < 15; ++a) { Hm[a] = T(0); }
	}
	if constexpr (KIND == kFinal) {
		#pragma unroll
		for (int a = 0; a < 15; ++a) { Fm[a] = T(0); }
	}
	T P1[3] = {T(0), T(0), T(0)}, P2[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
	if constexpr (MODEL == 8) {
		const T X0 = T((mp.sx - 1) * 0.5), Y0 = T((mp.sy - 1) * 0.5);
		int i = gl / roi, j = gl - i * roi;
		const int di = L / roi, dj = L - di * roi;
		for (int k = gl; k < n; k += L) {
			const T d = Photons<T>(px, i, j, k);
			const T psf = SplinePixel<T, NF>(mp, X0 + T(j - h) - th[2], Y0 + T(i - h) - th[3], th[4], P1, P2);
			Accumulate<T, KIND>(d, th[0], th[1], psf, P1, P2, D, G, Hm, Fm);
			i += di;
			j += dj;
			if (j >= roi) { j -= roi; ++i; }
		}
	}
	else if constexpr (L == 1) {
		const AxisConst<T> cx(sx), cy(sy);
		Bound<T> bp = MakeBound<T, NF>(0, h, th[2], cx.k);
		for (int c = 0; c < roi; ++c) {
			const Bound<T> bn = MakeBound<T, NF>(c + 1, h, th[2], cx.k);
			xt.template Put<NF>(c, FacOf<T, NF>(bp, bn, cx));
			bp = bn;
		}
		bp = MakeBound<T, NF>(0, h, th[3], cy.k);
		int k = 0;
		for (int i = 0; i < roi; ++i) {
			const Bound<T> bn = MakeBound<T, NF>(i + 1, h, th[3], cy.k);
			const Fac<T> yf = FacOf<T, NF>(bp, bn, cy);
			bp = bn;
			for (int j = 0; j < roi; ++j, ++k) {
				const T d = Photons<T>(px, i, j, k);
				const T psf = GaussPixel<T, NF>(xt.template Get<NF>(j), yf, dsx, dsy, ssx, ssy, P1, P2);
				Accumulate<T, KIND>(d, th[0], th[1], psf, P1, P2, D, G, Hm, Fm);
			}
		}
	}
	else if constexpr (L < 32) {
		// factor c of the columns (q = c) or the rows (q = roi + c) by lane q mod L, from its two boundaries
		const AxisConst<T> cx(sx), cy(sy);
		for (int q = gl; q < 2 * roi; q += L) {
			const bool isY = q >= roi;
			const int c = isY ? q - roi : q;
			const AxisConst<T>& ac = isY ? cy : cx;
			const T pos = isY ? th[3] : th[2];
			const Bound<T> a = MakeBound<T, NF>(c, h, pos, ac.k), b = MakeBound<T, NF>(c + 1, h, pos, ac.k);
			(isY ? yt : xt).template Put<NF>(c, FacOf<T, NF>(a, b, ac));
		}
		__syncwarp(GroupMask<L>());
		int i = gl / roi, j = gl - i * roi;
		const int di = L / roi, dj = L - di * roi;
		for (int k = gl; k < n; k += L) {
			const T d = Photons<T>(px, i, j, k);
			const T psf = GaussPixel<T, NF>(xt.template Get<NF>(j), yt.template Get<NF>(i), dsx, dsy, ssx, ssy, P1, P2);
			Accumulate<T, KIND>(d, th[0], th[1], psf, P1, P2, D, G, Hm, Fm);
			i += di;
			j += dj;
			if (j >= roi) { j -= roi; ++i; }
		}
		__syncwarp(GroupMask<L>());  // the tables are rewritten by the next evaluation
	}
	else {
		// lanes 0..roi hold the x boundaries, lanes 16..16+roi the y boundaries; pixel factors from lane pairs
		const AxisConst<T> cx(sx), cy(sy);
		const bool isY = gl >= 16;
		const int u = isY ? gl - 16 : gl;
		Bound<T> b{T(0), T(0), T(0), T(0), T(0)};
		if (u <= roi) { b = isY ? MakeBound<T, NF>(u, h, th[3], cy.k) : MakeBound<T, NF>(u, h, th[2], cx.k); }
		Bound<T> bn;
		bn.E = __shfl_down_sync(0xffffffffu, b.E, 1);
		bn.Q0 = __shfl_down_sync(0xffffffffu, b.Q0, 1);
		bn.Q1 = __shfl_down_sync(0xffffffffu, b.Q1, 1);
		bn.Q2 = __shfl_down_sync(0xffffffffu, b.Q2, 1);
		bn.Q3 = __shfl_down_sync(0xffffffffu, b.Q3, 1);
		if (u < roi) {
			if (isY) { yt.template Put<NF>(u, FacOf<T, NF>(b, bn, cy)); }
			else { xt.template Put<NF>(u, FacOf<T, NF>(b, bn, cx)); }
		}
		__syncwarp();
		int i = gl / roi, j = gl - i * roi;
		const int di = L / roi, dj = L - di * roi;
		for (int k = gl; k < n; k += L) {
			const T d = Photons<T>(px, i, j, k);
			const T psf = GaussPixel<T, NF>(xt.template Get<NF>(j), yt.template Get<NF>(i), dsx, dsy, ssx, ssy, P1, P2);
			Accumulate<T, KIND>(d, th[0], th[1], psf, P1, P2, D, G, Hm, Fm);
			i += di;
			j += dj;
			if (j >= roi) { j -= roi; ++i; }
		}
		__syncwarp();  // the tables are rewritten by the next evaluation
	}
	if constexpr (L > 1) {
		D = GroupSum<L>(D);
		if constexpr (KIND == kFisher || KIND == kExact) {
			#pragma unroll
			for (int a = 0; a < 5; ++a) { G[a] = GroupSum<L>(G[a]); }
			#pragma unroll
			for (int a = 0; a < 15; ++a) { Hm[a] = GroupSum<L>(Hm[a]); }
		}
		if constexpr (KIND == kFinal) {
			#pragma unroll
			for (int a = 0; a < 15; ++a) { Fm[a] = GroupSum<L>(Fm[a]); }
		}
	}
	return D;
}

__device__ __forceinline__ int Ut(int a, int b) { return a <= b ? a * 5 - (a * (a - 1)) / 2 + (b - a) : b * 5 - (b * (b - 1)) / 2 + (a - b); }

// Cholesky solve of the packed symmetric system (upper triangle) with the diagonal multiplied by diagScale. The pivot
// ratio is min_i L_ii^2 / A_ii: the pivots of the Jacobi-equilibrated system (unit diagonal), so it measures the
// conditioning independently of the parameters' units (photons, pixels, nm); 1 for a diagonal system.
template <typename T>
__device__ bool Chol5(const T Hm[15], T diagScale, const T rhs[5], T x[5], T* pivotRatio)
{
	T Lm[5][5];
	T minRatio = T(1);
	#pragma unroll
	for (int i = 0; i < 5; ++i) {
		#pragma unroll
		for (int j = 0; j <= i; ++j) {
			T s = Hm[Ut(i, j)];
			const T diag = s * diagScale;
			if (i == j) { s = diag; }
			#pragma unroll
			for (int k = 0; k < j; ++k) { s -= Lm[i][k] * Lm[j][k]; }
			if (i == j) {
				if (!(s > T(0))) { return false; }
				minRatio = min(minRatio, s / diag);
				Lm[i][i] = sqrt(s);
			}
			else { Lm[i][j] = s / Lm[j][j]; }
		}
	}
	T y[5];
	#pragma unroll
	for (int i = 0; i < 5; ++i) {
		T s = rhs[i];
		#pragma unroll
		for (int k = 0; k < i; ++k) { s -= Lm[i][k] * y[k]; }
		y[i] = s / Lm[i][i];
	}
	#pragma unroll
	for (int i = 4; i >= 0; --i) {
		T s = y[i];
		#pragma unroll
		for (int k = i + 1; k < 5; ++k) { s -= Lm[k][i] * x[k]; }
		x[i] = s / Lm[i][i];
	}
	if (pivotRatio) { *pivotRatio = minRatio; }
	return true;
}

// Diagonal of the inverse of the packed symmetric matrix F (upper triangle): one Cholesky factorisation F = L L^T,
// M = L^-1 by forward substitution with the reciprocal pivots, and (F^-1)_aa = sum_i M_ia^2. False when a pivot is not
// positive (the failure rule of Chol5).
template <typename T>
__device__ bool InverseDiag5(const T Fm[15], T out[5])
{
	T L[5][5], d[5];
	#pragma unroll
	for (int i = 0; i < 5; ++i) {
		#pragma unroll
		for (int j = 0; j <= i; ++j) {
			T s = Fm[Ut(i, j)];
			#pragma unroll
			for (int k = 0; k < j; ++k) { s -= L[i][k] * L[j][k]; }
			if (i == j) {
				if (!(s > T(0))) { return false; }
				L[i][i] = sqrt(s);
				d[i] = T(1) / L[i][i];
			}
			else { L[i][j] = s * d[j]; }
		}
	}
	T M[5][5];
	#pragma unroll
	for (int j = 0; j < 5; ++j) {
		M[j][j] = d[j];
		#pragma unroll
		for (int i = j + 1; i < 5; ++i) {
			T s = T(0);
			#pragma unroll
			for (int k = j; k < i; ++k) { s += L[i][k] * M[k][j]; }
			M[i][j] = -s * d[i];
		}
	}
	#pragma unroll
	for (int a = 0; a < 5; ++a) {
		T v = T(0);
		#pragma unroll
		for (int i = a; i < 5; ++i) { v += M[i][a] * M[i][a]; }
		out[a] = v;
	}
	return true;
}

// FP32 solve of (Hm with its diagonal scaled) dt = rhs; re-factored in FP64 when the FP32 factorisation fails or its
// pivot ratio is below 1e-5, i.e. when elimination cancelled more than 5 of the 7 significant digits of FP32 in some
// pivot (counted in *fallbacks when count is set).
__device__ bool Solve32(const float Hm[15], float scale, const float rhs[5], float dt[5], unsigned* fallbacks, bool count)
{
	float ratio = 0.f;
	if (Chol5<float>(Hm, scale, rhs, dt, &ratio) && ratio >= 1e-5f) { return true; }
	double Hd[15], rd[5], xd[5];
	#pragma unroll
	for (int a = 0; a < 15; ++a) { Hd[a] = Hm[a]; }
	#pragma unroll
	for (int a = 0; a < 5; ++a) { rd[a] = rhs[a]; }
	const bool ok = Chol5<double>(Hd, static_cast<double>(scale), rd, xd, nullptr);
	if (count && fallbacks) { atomicAdd(fallbacks, 1u); }
	#pragma unroll
	for (int a = 0; a < 5; ++a) { dt[a] = static_cast<float>(xd[a]); }
	return ok;
}

// Bounds of theta (MleBounds in the oracle); x0, y0 = candidate position relative to the ROI centre.
template <int MODEL>
__device__ __forceinline__ void Bounds(const MleParams& mp, double x0, double y0, double lo[5], double hi[5])
{
	const double hf = static_cast<double>(mp.half);
	lo[0] = 1e-3; hi[0] = 1e6;
	lo[1] = 1.0; hi[1] = 1e9;
	lo[2] = fmax(x0 - 2.0, -hf); hi[2] = fmin(x0 + 2.0, hf);
	lo[3] = fmax(y0 - 2.0, -hf); hi[3] = fmin(y0 + 2.0, hf);
	if (MODEL == 6) { lo[4] = 0.5; hi[4] = 5.0; }
	else if (MODEL == 7) { lo[4] = mp.zMin; hi[4] = mp.zMax; }
	else { lo[4] = 0.0; hi[4] = static_cast<double>(mp.sz) - 1e-6; }
}

// The same bounds in FP32 (the spline's upper z bound is the largest float below sz).
template <int MODEL>
__device__ __forceinline__ void Bounds32(const MleParams& mp, float x0, float y0, float lo[5], float hi[5])
{
	const float hf = static_cast<float>(mp.half);
	lo[0] = 1e-3f; hi[0] = 1e6f;
	lo[1] = 1.f; hi[1] = 1e9f;
	lo[2] = fmaxf(x0 - 2.f, -hf); hi[2] = fminf(x0 + 2.f, hf);
	lo[3] = fmaxf(y0 - 2.f, -hf); hi[3] = fminf(y0 + 2.f, hf);
	if (MODEL == 6) { lo[4] = 0.5f; hi[4] = 5.f; }
	else if (MODEL == 7) { lo[4] = static_cast<float>(mp.zMin); hi[4] = static_cast<float>(mp.zMax); }
	else { lo[4] = 0.f; hi[4] = nextafterf(static_cast<float>(mp.sz), 0.f); }
}

template <int MODEL>
__device__ __forceinline__ void Clamp32(const MleParams& mp, float x0, float y0, float t[5])
{
	float lo[5], hi[5];
	Bounds32<MODEL>(mp, x0, y0, lo, hi);
	#pragma unroll
	for (int a = 0; a < 5; ++a) { t[a] = fminf(fmaxf(t[a], lo[a]), hi[a]); }
}

// Active bounds (FixActive in the oracle): a parameter on a bound whose descent direction -G points outside is held
// there - its row and column of the packed system become those of the identity, its right-hand side zero.
template <int MODEL>
__device__ __forceinline__ void FixActive32(const MleParams& mp, float x0, float y0, const float t[5], const float G[5], float A[15],
                                            float rhs[5])
{
	float lo[5], hi[5];
	Bounds32<MODEL>(mp, x0, y0, lo, hi);
	#pragma unroll
	for (int a = 0; a < 5; ++a) {
		if ((t[a] <= lo[a] && G[a] > 0.f) || (t[a] >= hi[a] && G[a] < 0.f)) {
			#pragma unroll
			for (int b = 0; b < 5; ++b) { A[Ut(a, b)] = 0.f; }
			A[Ut(a, a)] = 1.f;
			rhs[a] = 0.f;
		}
	}
}

// LM stop rule: the oracle's (MleStepSmall: 1e-4 px in x and y, 1e-4 relative in I and bg with floor 1, 1e-4 for
// sigma and the spline z, 1e-2 nm for z) with every threshold multiplied by kLmStepScale. The FP32 deviance cannot
// resolve the last LM steps of the oracle (a 1e-4 px step changes the deviance by about 1e-5, the size of its FP32
// rounding), so the FP32 LM hands over to the Newton polish earlier (a 3e-2 px step): the polish converges
// quadratically from there to the same optimum. Measured on the 2000-frame benchmark (LM / polish evaluations, fit
// stage, step): 10x 36.9 M / 15.1 M; 100x 24.2 M / 11.6 M, 16.9 ms, 41.9 ms; 300x 21.2 M / 12.5 M, 16.6 ms,
// 41.5 ms; 1000x 17.9 M / 14.2 M, 16.5 ms, 41.5 ms; the same error table throughout.
constexpr float kLmStepScale = 300.f;
__device__ __forceinline__ bool StepSmall(int model, const float a[5], const float b[5])
{
	const float t = 1e-4f * kLmStepScale, sTol = (model == 7 ? 1e-2f : 1e-4f) * kLmStepScale;
	return fabsf(b[2] - a[2]) < t && fabsf(b[3] - a[3]) < t && fabsf(b[1] - a[1]) < t * fmaxf(fabsf(a[1]), 1.f) &&
	       fabsf(b[0] - a[0]) < t * fmaxf(fabsf(a[0]), 1.f) && fabsf(b[4] - a[4]) < sTol;
}

// Newton direction at th: the exact Hessian with active bounds held, Fisher scoring where that Hessian is not
// positive definite. Hm is modified in place. fisher(Hf) fills Hf with the Fisher-scoring matrix 2 F at th (an extra
// evaluation, made only in that case).
template <int MODEL, typename FisherFn>
__device__ __forceinline__ bool NewtonDirection(const MleParams& mp, float x0, float y0, const float th[5], const float G[5], float Hm[15],
                                                float dt[5], FisherFn fisher)
{
	float rhs[5];
	#pragma unroll
	for (int a = 0; a < 5; ++a) { rhs[a] = -G[a]; }
	FixActive32<MODEL>(mp, x0, y0, th, G, Hm, rhs);
	if (Solve32(Hm, 1.f, rhs, dt, nullptr, false)) { return true; }
	float Hf[15];
	fisher(Hf);
	FixActive32<MODEL>(mp, x0, y0, th, G, Hf, rhs);
	return Solve32(Hf, 1.f, rhs, dt, nullptr, false);
}

// Newton polish acceptance: the trial deviance may exceed the current one by its FP32 rounding (steps near the
// optimum change the deviance by less than that).
__device__ __forceinline__ bool PolishAccept(float Dt, float D) { return isfinite(Dt) && Dt <= D + 1e-5f * (fabsf(D) + 1.f); }

// ROI geometry of a candidate; false when the ROI crosses the frame border (the reference's test, Fitting.cpp).
struct RoiAt {
	unsigned long long ux, uy;
	double x0, y0;
	const uint16_t* base;
	int W;  // row pitch of the ROI's frame
};

__device__ __forceinline__ bool Locate(const FitImages& fi, const MleParams& mp, const Cand& cd, RoiAt& r)
{
	const FitImage& f = fi.im[cd.image];
	const int H = f.H, W = f.W;
	r.W = W;
	const bool nonneg = cd.x >= 0.0 && cd.y >= 0.0;
	r.ux = nonneg ? static_cast<unsigned long long>(cd.x) : 0ull;
	r.uy = nonneg ? static_cast<unsigned long long>(cd.y) : 0ull;
	const unsigned long long hh = static_cast<unsigned long long>(mp.half);
	if (!nonneg || hh > r.ux || r.ux >= static_cast<unsigned long long>(W) - hh || hh > r.uy || r.uy >= static_cast<unsigned long long>(H) - hh) {
		return false;
	}
	r.x0 = cd.x - static_cast<double>(r.ux);
	r.y0 = cd.y - static_cast<double>(r.uy);
	r.base = f.img + static_cast<long long>(cd.frame) * f.N + static_cast<long long>(r.uy - hh) * W + static_cast<long long>(r.ux - hh);
	return true;
}

__device__ __forceinline__ Pix MakePix(const MleParams& mp, const uint16_t* base, int W, const float* sm, int ss)
{
	Pix p;
	p.sm = sm;
	p.ss = ss;
	p.g = base;
	p.W = W;
	p.off32 = static_cast<float>(mp.offset);
	p.inv32 = static_cast<float>(1.0 / mp.gain);
	p.off64 = mp.offset;
	p.inv64 = 1.0 / mp.gain;
	return p;
}

// Initial values (oracle MleFit): bg = min photons (>= 1e-3), I = photons above bg (>= 1), x, y = candidate, s =
// sigma0 (mode 6) or the best of a deviance scan of the axial range (16 points for mode 7, 8 for mode 8). The oracle
// scans in FP64; here the scan runs in FP32 like the LM it starts (its choice differs only where two grid points'
// deviances agree to FP32 rounding, and the LM then descends into the same basin). xt, yt: FP32 factor tables.
template <int MODEL, int L>
__device__ int InitTheta(const MleParams& mp, const Pix& px, const RoiAt& r, double t[5], FacTab<float> xt, FacTab<float> yt)
{
	int evals = 0;
	const int gl = L == 1 ? 0 : (threadIdx.x & 31);
	double dmin = 1e300, sum = 0;
	for (int k = gl; k < mp.n; k += L) {
		const int i = k / mp.roi, j = k - i * mp.roi;
		const double d = Photons<double>(px, i, j, k);
		dmin = fmin(dmin, d);
		sum += d;
	}
	if constexpr (L > 1) {
		#pragma unroll
		for (int d = 16; d > 0; d >>= 1) {
			dmin = fmin(dmin, __shfl_xor_sync(0xffffffffu, dmin, d));
			sum += __shfl_xor_sync(0xffffffffu, sum, d);
		}
	}
	double lo[5], hi[5];
	Bounds<MODEL>(mp, r.x0, r.y0, lo, hi);
	t[0] = fmax(dmin, 1e-3);
	t[1] = fmax(sum - t[0] * mp.n, 1.0);
	t[2] = r.x0;
	t[3] = r.y0;
	if (MODEL == 6) { t[4] = mp.sigma0; }
	else {
		const int ns = MODEL == 7 ? 16 : 8;
		float best = __int_as_float(0x7f800000), tf[5] = {float(t[0]), float(t[1]), float(t[2]), float(t[3]), 0.f};
		double bz = 0.5 * (lo[4] + hi[4]);
		for (int s = 0; s < ns; ++s) {
			const double z = lo[4] + (hi[4] - lo[4]) * (s + 0.5) / ns;
			tf[4] = float(z);
			const float D = Normal<float, MODEL, L, kDevOnly>(mp, px, tf, nullptr, nullptr, nullptr, xt, yt);
			++evals;
			if (D < best) { best = D; bz = z; }
		}
		t[4] = bz;
	}
	#pragma unroll
	for (int a = 0; a < 5; ++a) { t[a] = fmin(fmax(t[a], lo[a]), hi[a]); }
	return evals;
}

// A Newton step below the polish's 1e-6 relative stop is applied without evaluating the deviance there: the
// evaluation could only confirm a change below the FP32 resolution of the parameters.
template <int MODEL>
__device__ __forceinline__ bool ApplyIfTiny(const MleParams& mp, float x0, float y0, float th[5], const float dt[5])
{
	float step = 0.f;
	#pragma unroll
	for (int a = 0; a < 5; ++a) { step = fmaxf(step, fabsf(dt[a]) / fmaxf(fabsf(th[a]), 1.f)); }
	if (!(step < 1e-6f)) { return false; }
	#pragma unroll
	for (int a = 0; a < 5; ++a) { th[a] += dt[a]; }
	Clamp32<MODEL>(mp, x0, y0, th);
	return true;
}

// FP32 Newton steps on the exact Hessian of the deviance (NewtonDirection), at most 6; a step that the deviance does
// not accept (PolishAccept) is halved up to three times; stops at a 1e-6 relative step (the oracle: FP64, 1e-10).
template <int MODEL, int L>
__device__ int Polish(const MleParams& mp, const Pix& px, float x0, float y0, float th[5], FacTab<float> xt, FacTab<float> yt)
{
	float G[5], Hm[15];
	float D = Normal<float, MODEL, L, kExact>(mp, px, th, G, Hm, nullptr, xt, yt);
	int evals = 1;
	if (!isfinite(D)) { return evals; }
	for (int it = 0; it < 6; ++it) {
		float dt[5], tt[5];
		auto fisher = [&](float Hf[15]) {
			float Gf[5];
			Normal<float, MODEL, L, kFisher>(mp, px, th, Gf, Hf, nullptr, xt, yt);
			++evals;
		};
		if (!NewtonDirection<MODEL>(mp, x0, y0, th, G, Hm, dt, fisher)) { break; }
		if (ApplyIfTiny<MODEL>(mp, x0, y0, th, dt)) { break; }
		bool accepted = false;
		float Gt[5], Ht[15], Dt = 0.f;
		for (int hv = 0; hv < 4 && !accepted; ++hv) {
			#pragma unroll
			for (int a = 0; a < 5; ++a) { tt[a] = th[a] + dt[a]; }
			Clamp32<MODEL>(mp, x0, y0, tt);
			Dt = Normal<float, MODEL, L, kExact>(mp, px, tt, Gt, Ht, nullptr, xt, yt);
			++evals;
			if (PolishAccept(Dt, D)) { accepted = true; }
			else {
				#pragma unroll
				for (int a = 0; a < 5; ++a) { dt[a] *= 0.5f; }
			}
		}
		if (!accepted) { break; }
		float step = 0.f;
		#pragma unroll
		for (int a = 0; a < 5; ++a) { step = fmaxf(step, fabsf(tt[a] - th[a]) / fmaxf(fabsf(th[a]), 1.f)); }
		#pragma unroll
		for (int a = 0; a < 5; ++a) { th[a] = tt[a]; G[a] = Gt[a]; }
		#pragma unroll
		for (int a = 0; a < 15; ++a) { Hm[a] = Ht[a]; }
		D = Dt;
		if (step < 1e-6f) { break; }
	}
	return evals;
}

// FP64 final pass at t: the Poisson deviance D (the log-likelihood ratio against the saturated model, -2 log(L/L_sat),
// the fit's goodness of fit) and the Fisher information; CRLB = sqrt(diag(F^-1)). False when F cannot be inverted or t
// is not finite (the oracle's final step).
template <int MODEL, int L>
__device__ bool Final(const MleParams& mp, const Pix& px, const double t[5], double crlb[5], double& dev, FacTab<double> xt,
                      FacTab<double> yt)
{
	double Fm[15], cv[5];
	dev = Normal<double, MODEL, L, kFinal>(mp, px, t, nullptr, nullptr, Fm, xt, yt);  // a non-finite entry fails the Cholesky
	if (!InverseDiag5<double>(Fm, cv)) { return false; }
	#pragma unroll
	for (int a = 0; a < 5; ++a) { crlb[a] = cv[a] > 0 ? sqrt(cv[a]) : 0.0; }
	#pragma unroll
	for (int a = 0; a < 5; ++a) {
		if (!isfinite(t[a])) { return false; }
	}
	return true;
}

// Output row; col < 0: the calling thread writes all 18 columns, else only column col. The Theta column (the models
// have no rotation) holds the FP64 deviance of the fit, -1 for a failed one.
__device__ void StoreMleRow(double* row, int col, const MleParams& mp, const Cand& cd, const double t[5], const double crlb[5],
                            double dev, unsigned long long ux, unsigned long long uy, bool ok)
{
	double v[kCols];
	v[cId] = 0; v[cPlane] = 0; v[cIndex] = 0; v[cChannel] = -1;
	const double qxy = sqrt(0.5 * (crlb[2] * crlb[2] + crlb[3] * crlb[3]));
	if (ok && mp.crlbMax > 0 && !(qxy <= mp.crlbMax)) { ok = false; }
	if (!ok) {
		v[cX] = cd.x; v[cY] = cd.y; v[cZ] = 0; v[cIntensity] = -1; v[cSigmaX] = -1; v[cSigmaY] = -1; v[cTheta] = -1;
		v[cQualityXY] = -1; v[cQualityZ] = -1; v[cAmplitude] = -1; v[cOffset] = -1; v[cCircularity] = 1;
	}
	else {
		double sx = t[4], sy = t[4], z = 0, qz = -1;
		if (mp.model == 7) {
			double d1, d2;
			AstigSigma<double>(mp.astig, mp.pixelSize, t[4], sx, d1, d2);
			AstigSigma<double>(mp.astig + 5, mp.pixelSize, t[4], sy, d1, d2);
			z = t[4];
			qz = crlb[4];
		}
		if (mp.model == 8) { sx = sy = 0; z = mp.dz * (t[4] - mp.sz / 2.0); qz = mp.dz * crlb[4]; }
		v[cX] = static_cast<double>(ux) + t[2];
		v[cY] = static_cast<double>(uy) + t[3];
		v[cZ] = z;
		v[cIntensity] = t[1];
		v[cSigmaX] = sx; v[cSigmaY] = sy; v[cTheta] = dev;
		v[cQualityXY] = qxy; v[cQualityZ] = qz;
		v[cAmplitude] = (sx > 0 && sy > 0) ? t[1] / (6.283185307179586 * sx * sy) : t[1];
		v[cOffset] = t[0];
		v[cCircularity] = (sx > kEps && sy > kEps) ? fmin(sx, sy) / fmax(sx, sy) : 1;
	}
	v[cSegIntensity] = cd.intensity; v[cSurface] = cd.surf;
	if (col < 0) {
		#pragma unroll
		for (int c = 0; c < kCols; ++c) { row[c] = v[c]; }
	}
	else {
		#pragma unroll
		for (int c = 0; c < kCols; ++c) {
			if (col == c) { row[c] = v[c]; }
		}
	}
}

__device__ __forceinline__ uint32_t CandCount(const uint32_t* nptr, uint32_t nconst) { return nptr ? *nptr : nconst; }

// ---------------------------------------------------------------------------------------------------------------
// Thread per ROI.

// Initial values; shared memory: per thread the FP32 column factors of the axial pre-scan (roi floats).
template <int MODEL>
__global__ void __launch_bounds__(kThreads) MleInitKernel(FitImages fi,
                                                          const Cand* __restrict__ cands, const uint32_t* nptr, uint32_t nconst,
                                                          MleParams mp, double* rows)
{
	extern __shared__ __align__(16) unsigned char smem[];
	const FacTab<float> xt{reinterpret_cast<float*>(smem) + threadIdx.x, static_cast<int>(blockDim.x)};
	const uint32_t n = CandCount(nptr, nconst);
	unsigned long long evals = 0;
	for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
		double* row = rows + static_cast<long long>(k) * kCols;
		RoiAt r;
		if (!Locate(fi, mp, cands[k], r)) {
			row[kStatusCol] = kStBorder;
			continue;
		}
		const Pix px = MakePix(mp, r.base, r.W, nullptr, 0);
		double t[5];
		evals += InitTheta<MODEL, 1>(mp, px, r, t, xt, xt);
		#pragma unroll
		for (int a = 0; a < 5; ++a) { row[a] = t[a]; }
		row[kStatusCol] = kStOk;
	}
	if (mp.evals && evals) { atomicAdd(mp.evals + 2, evals); }
}

constexpr uint32_t kNone = 0xffffffffu;

// Work queue of the persistent kernels. With a counter (zeroed before the launch) it is global: lanes that need work
// take the next candidates with one atomic per warp, so warps that finish early keep taking work until all
// candidates are out; each taking lane receives `chunk` consecutive candidates (neighbouring ROIs of one frame) and
// starts the next of them without an atomic. Without a counter, warp w owns the static range
// [w * c, (w + 1) * c), c >= 32.
struct WarpQueue {
	uint32_t cursor, end, chunk;
	uint32_t next, last;  // this lane's taken candidates not started yet: [next, last)
	unsigned int* counter;
	__device__ __forceinline__ bool Init(uint32_t n, unsigned int* ctr, int chunkSize)
	{
		counter = ctr;
		chunk = static_cast<uint32_t>(max(chunkSize, 1));
		next = last = 0;
		if (counter) {
			cursor = 0;
			end = n;
			return n > 0;
		}
		const uint32_t warps = gridDim.x * (blockDim.x / 32);
		const uint32_t gw = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
		const uint32_t c = max(32u, (n + warps - 1) / warps);
		const unsigned long long begin = static_cast<unsigned long long>(gw) * c;
		cursor = static_cast<uint32_t>(min(begin, static_cast<unsigned long long>(n)));
		end = static_cast<uint32_t>(min(begin + c, static_cast<unsigned long long>(n)));
		return cursor < end;
	}
	// Called by all 32 lanes; returns the candidate taken by a lane with `need` set (kNone when the queue is done).
	__device__ __forceinline__ uint32_t Take(bool need)
	{
		const int lane = threadIdx.x & 31;
		if (counter) {
			const bool fetch = need && next >= last;
			const unsigned mask = __ballot_sync(0xffffffffu, fetch);
			if (mask != 0 && cursor < end) {
				const int leader = __ffs(mask) - 1;
				const uint32_t want = static_cast<uint32_t>(__popc(mask)) * chunk;
				uint32_t base = 0;
				if (lane == leader) { base = atomicAdd(counter, want); }
				base = __shfl_sync(0xffffffffu, base, leader);
				if (base + want >= end) { cursor = end; }  // the queue ran out: stop taking
				if (fetch) {
					next = min(base + __popc(mask & ((1u << lane) - 1u)) * chunk, end);
					last = min(next + chunk, end);
				}
			}
			return need && next < last ? next++ : kNone;
		}
		const unsigned mask = __ballot_sync(0xffffffffu, need);
		const uint32_t k = cursor + __popc(mask & ((1u << lane) - 1u));
		cursor = min(end, cursor + static_cast<uint32_t>(__popc(mask)));
		return need && k < end ? k : kNone;
	}
	// Called by all 32 lanes: nothing left to take, neither in the queue nor in any lane's chunk.
	__device__ __forceinline__ bool Done() const { return cursor >= end && __ballot_sync(0xffffffffu, next < last) == 0; }
};

// The calling lane's share of a group of L lanes that handles one ROI: its index in the group, the group's first lane
// and whether it is that lane (which takes the queue's candidates, counts and writes the rows).
template <int L>
struct Group {
	int gl, first;
	bool leader;
	__device__ __forceinline__ Group()
	{
		const int lane = threadIdx.x & 31;
		gl = lane & (L - 1);
		first = lane - gl;
		leader = gl == 0;
	}
};

// Stages the ROI of candidate k: FP32 photons at ph[q * T] (the L lanes of a group share the pixels), theta from the
// row, position.
template <int L>
__device__ __forceinline__ void LoadRoi(const FitImages& fi, const MleParams& mp, const Cand* cands, const double* rows, uint32_t k,
                                        float* ph, int T, Pix& px, float th[5], float& x0, float& y0)
{
	RoiAt r;
	Locate(fi, mp, cands[k], r);
	const int W = r.W;
	px.g = r.base;
	px.W = W;
	const int gl = L == 1 ? 0 : static_cast<int>(threadIdx.x & (L - 1));
	for (int q = gl; q < mp.n; q += L) {
		const int i = q / mp.roi, j = q - i * mp.roi;
		ph[q * T] = fmaxf((float(__ldg(r.base + i * W + j)) - px.off32) * px.inv32, 0.f);
	}
	if constexpr (L > 1) { __syncwarp(GroupMask<L>()); }
	const double* row = rows + static_cast<long long>(k) * kCols;
	#pragma unroll
	for (int a = 0; a < 5; ++a) { th[a] = static_cast<float>(row[a]); }
	x0 = static_cast<float>(r.x0);
	y0 = static_cast<float>(r.y0);
}

// Shared memory of the persistent kernels per ROI slot, in floats: the photons and the column (and, for L > 1, row)
// factor tables with NF fields. L = 1: lane-interleaved slots (stride = block size); L > 1: one contiguous slot per
// group.
__host__ __device__ __forceinline__ int SlotFloats(int n, int roi, int nf, int L) { return n + (L == 1 ? 1 : 2) * nf * roi; }

template <int L>
struct SlotView {
	float* ph;
	int stride;
	FacTab<float> xt, yt;
	__device__ __forceinline__ SlotView(unsigned char* smem, const MleParams& mp, int nf)
	{
		float* base = reinterpret_cast<float*>(smem);
		if constexpr (L == 1) {
			const int T = blockDim.x;
			ph = base + threadIdx.x;
			stride = T;
			xt = FacTab<float>{base + mp.n * T + threadIdx.x, T};
			yt = xt;
		}
		else {
			float* slot = base + (threadIdx.x / L) * SlotFloats(mp.n, mp.roi, nf, L);
			ph = slot;
			stride = 1;
			xt = FacTab<float>{slot + mp.n, 1};
			yt = FacTab<float>{slot + mp.n + nf * mp.roi, 1};
		}
	}
};

// Persistent FP32 LM (WarpQueue). Every pass of the loop makes each busy ROI evaluate the deviance, gradient and
// Fisher matrix once: at the start point of a new candidate, or at the trial point of an LM step. L lanes per ROI
// (1: a thread per ROI); the lanes of a group hold the same state and take the same branches. Shared memory per ROI
// slot: the photons and the factor tables (SlotFloats, NF = 3).
template <int MODEL, int L>
__global__ void __launch_bounds__(kThreads) MleLmKernel(FitImages fi,
                                                        const Cand* __restrict__ cands, const uint32_t* nptr, uint32_t nconst,
                                                        MleParams mp, double* rows)
{
	extern __shared__ __align__(16) unsigned char smem[];
	const SlotView<L> sv(smem, mp, 3);
	const Group<L> grp;
	WarpQueue q;
	if (!q.Init(CandCount(nptr, nconst), mp.queue, mp.chunk)) { return; }
	uint32_t k = kNone;
	bool fresh = false;
	float th[5] = {0, 0, 0, 0, 0}, G[5], Hm[15], D = 0.f, lambda = 1e-3f, x0 = 0.f, y0 = 0.f;
	int it = 0;
	unsigned long long evals = 0;
	Pix px = MakePix(mp, nullptr, 0, sv.ph, sv.stride);
	while (true) {
		uint32_t kk = q.Take(grp.leader && k == kNone);
		if constexpr (L > 1) { kk = __shfl_sync(0xffffffffu, kk, grp.first); }
		if (kk != kNone && rows[static_cast<long long>(kk) * kCols + kStatusCol] == kStOk) {
			LoadRoi<L>(fi, mp, cands, rows, kk, sv.ph, sv.stride, px, th, x0, y0);
			k = kk;
			fresh = true;
		}
		const bool busy = k != kNone;
		if (__ballot_sync(0xffffffffu, busy) == 0) {
			if (q.Done()) { break; }
			continue;
		}
		float tt[5];
		bool eval = false, finish = false, failed = false;
		if (busy) {
			if (fresh) {
				#pragma unroll
				for (int a = 0; a < 5; ++a) { tt[a] = th[a]; }
				eval = true;
			}
			else {
				float rhs[5], dt[5];
				#pragma unroll
				for (int a = 0; a < 5; ++a) { rhs[a] = -G[a]; }
				FixActive32<MODEL>(mp, x0, y0, th, G, Hm, rhs);  // in place: Hm is replaced when a step is accepted
				if (Solve32(Hm, 1.f + lambda, rhs, dt, mp.fallbacks, grp.leader)) {
					#pragma unroll
					for (int a = 0; a < 5; ++a) { tt[a] = th[a] + dt[a]; }
					Clamp32<MODEL>(mp, x0, y0, tt);
					eval = true;
				}
				else {
					++it;
					lambda *= 10.f;
					finish = lambda > 1e7f || it >= mp.maxIter;
				}
			}
		}
		float Gt[5], Ht[15], Dt = 0.f;
		if (eval) {
			Dt = Normal<float, MODEL, L, kFisher>(mp, px, tt, Gt, Ht, nullptr, sv.xt, sv.yt);
			evals += grp.leader ? 1 : 0;
			if (fresh) {
				fresh = false;
				D = Dt;
				#pragma unroll
				for (int a = 0; a < 5; ++a) { G[a] = Gt[a]; }
				#pragma unroll
				for (int a = 0; a < 15; ++a) { Hm[a] = Ht[a]; }
				lambda = 1e-3f;
				it = 0;
				failed = !isfinite(D);
				finish = failed || mp.maxIter <= 0;
			}
			else {
				++it;
				if (isfinite(Dt) && Dt < D) {
					const bool small = StepSmall(MODEL, th, tt);
					#pragma unroll
					for (int a = 0; a < 5; ++a) { th[a] = tt[a]; G[a] = Gt[a]; }
					#pragma unroll
					for (int a = 0; a < 15; ++a) { Hm[a] = Ht[a]; }
					D = Dt;
					lambda = fmaxf(lambda * 0.1f, 1e-7f);
					finish = small;
				}
				else {
					lambda *= 10.f;
					finish = lambda > 1e7f;
				}
				finish = finish || it >= mp.maxIter;
			}
		}
		if (finish) {
			if (grp.leader) {
				double* row = rows + static_cast<long long>(k) * kCols;
				#pragma unroll
				for (int a = 0; a < 5; ++a) { row[a] = th[a]; }
				row[kStatusCol] = failed ? kStFailed : kStOk;
			}
			k = kNone;
		}
	}
	if (mp.evals && evals) { atomicAdd(mp.evals, evals); }
}

// Persistent FP32 Newton polish (WarpQueue), the steps of Polish() as a per-ROI state machine: each pass evaluates
// the deviance, gradient and exact Hessian once per busy ROI - at the LM result of a new candidate or at a trial
// point - and then accepts, halves or ends. L lanes per ROI as in the LM. Shared memory per ROI slot: the photons and
// the factor tables with second derivatives (SlotFloats, NF = 6). Mode 6 with a thread per ROI is held to 128
// registers (8 blocks of 64 threads per SM instead of 6 at its own 150), which it fits without spilling.
template <int MODEL, int L>
__global__ void __launch_bounds__(kThreads, MODEL == 6 && L == 1 ? 8 : 0) MlePolishKernel(FitImages fi,
                                                            const Cand* __restrict__ cands, const uint32_t* nptr, uint32_t nconst,
                                                            MleParams mp, double* rows)
{
	extern __shared__ __align__(16) unsigned char smem[];
	const SlotView<L> sv(smem, mp, 6);
	const Group<L> grp;
	WarpQueue q;
	if (!q.Init(CandCount(nptr, nconst), mp.queue ? mp.queue + 1 : nullptr, mp.chunk)) { return; }
	uint32_t k = kNone;
	bool fresh = false;
	float th[5] = {0, 0, 0, 0, 0}, dt[5] = {0, 0, 0, 0, 0}, G[5], Hm[15], D = 0.f, x0 = 0.f, y0 = 0.f;
	int it = 0, hv = 0;
	unsigned long long evals = 0;
	Pix px = MakePix(mp, nullptr, 0, sv.ph, sv.stride);
	while (true) {
		uint32_t kk = q.Take(grp.leader && k == kNone);
		if constexpr (L > 1) { kk = __shfl_sync(0xffffffffu, kk, grp.first); }
		if (kk != kNone && rows[static_cast<long long>(kk) * kCols + kStatusCol] == kStOk) {
			LoadRoi<L>(fi, mp, cands, rows, kk, sv.ph, sv.stride, px, th, x0, y0);
			k = kk;
			fresh = true;
		}
		const bool busy = k != kNone;
		if (__ballot_sync(0xffffffffu, busy) == 0) {
			if (q.Done()) { break; }
			continue;
		}
		float tt[5], Gt[5], Ht[15], Dt = 0.f;
		bool finish = false;
		if (busy) {
			#pragma unroll
			for (int a = 0; a < 5; ++a) { tt[a] = fresh ? th[a] : th[a] + dt[a]; }
			if (!fresh) { Clamp32<MODEL>(mp, x0, y0, tt); }
			Dt = Normal<float, MODEL, L, kExact>(mp, px, tt, Gt, Ht, nullptr, sv.xt, sv.yt);
			evals += grp.leader ? 1 : 0;
			bool moved = false;
			if (fresh) {
				fresh = false;
				it = 0;
				moved = isfinite(Dt);
				finish = !moved;
			}
			else if (PolishAccept(Dt, D)) {
				float step = 0.f;
				#pragma unroll
				for (int a = 0; a < 5; ++a) { step = fmaxf(step, fabsf(tt[a] - th[a]) / fmaxf(fabsf(th[a]), 1.f)); }
				++it;
				finish = step < 1e-6f || it >= 6;
				moved = true;
			}
			else if (++hv >= 4) { finish = true; }
			else {
				#pragma unroll
				for (int a = 0; a < 5; ++a) { dt[a] *= 0.5f; }
			}
			if (moved) {
				#pragma unroll
				for (int a = 0; a < 5; ++a) { th[a] = tt[a]; G[a] = Gt[a]; }
				#pragma unroll
				for (int a = 0; a < 15; ++a) { Hm[a] = Ht[a]; }
				D = Dt;
				hv = 0;
				if (!finish) {
					auto fisher = [&](float Hf[15]) {
						float Gf[5];
						Normal<float, MODEL, L, kFisher>(mp, px, th, Gf, Hf, nullptr, sv.xt, sv.yt);
						evals += grp.leader ? 1 : 0;
					};
					finish = !NewtonDirection<MODEL>(mp, x0, y0, th, G, Hm, dt, fisher) || ApplyIfTiny<MODEL>(mp, x0, y0, th, dt);
				}
			}
		}
		if (finish) {
			if (grp.leader) {
				double* row = rows + static_cast<long long>(k) * kCols;
				#pragma unroll
				for (int a = 0; a < 5; ++a) { row[a] = th[a]; }
			}
			k = kNone;
		}
	}
	if (mp.evals && evals) { atomicAdd(mp.evals + 1, evals); }
}

// FP64 deviance, Fisher information and CRLB at the polished theta; writes the output row. Shared memory per thread:
// the FP64 column factors (3 roi doubles). Mode 6 is held to 128 registers (8 blocks of 64 threads per SM), which it
// fits without spilling; modes 7 and 8 keep the compiler's own allocation (a bound spills them).
template <int MODEL>
__global__ void __launch_bounds__(kThreads, MODEL == 6 ? 8 : 0) MleFinalKernel(FitImages fi,
                                                           const Cand* __restrict__ cands, const uint32_t* nptr, uint32_t nconst,
                                                           MleParams mp, double* rows)
{
	extern __shared__ __align__(16) unsigned char smem[];
	const FacTab<double> xt{reinterpret_cast<double*>(smem) + threadIdx.x, static_cast<int>(blockDim.x)};
	const uint32_t n = CandCount(nptr, nconst);
	unsigned long long evals = 0;
	for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
		double* row = rows + static_cast<long long>(k) * kCols;
		const Cand cd = cands[k];
		RoiAt r;
		double t[5] = {0, 0, 0, 0, 0}, crlb[5] = {0, 0, 0, 0, 0}, dev = 0;
		bool ok = Locate(fi, mp, cd, r) && row[kStatusCol] == kStOk;
		if (ok) {
			#pragma unroll
			for (int a = 0; a < 5; ++a) { t[a] = row[a]; }
			ok = Final<MODEL, 1>(mp, MakePix(mp, r.base, r.W, nullptr, 0), t, crlb, dev, xt, xt);
			++evals;
		}
		StoreMleRow(row, -1, mp, cd, t, crlb, dev, r.ux, r.uy, ok);
	}
	if (mp.evals && evals) { atomicAdd(mp.evals + 2, evals); }
}

// ---------------------------------------------------------------------------------------------------------------
// Warp per ROI: all phases in one launch.

struct WarpSmem {
	float photons[kMaxPix];
	double xt[6 * kMaxRoi];
	double yt[6 * kMaxRoi];
};

template <int MODEL>
__global__ void __launch_bounds__(kThreads) MleWarpKernel(FitImages fi,
                                                          const Cand* __restrict__ cands, const uint32_t* nptr, uint32_t nconst,
                                                          MleParams mp, double* rows)
{
	__shared__ WarpSmem sm[kThreads / 32];
	WarpSmem& ws = sm[threadIdx.x / 32];
	const FacTab<float> xt32{reinterpret_cast<float*>(ws.xt), 1}, yt32{reinterpret_cast<float*>(ws.yt), 1};
	const FacTab<double> xt64{ws.xt, 1}, yt64{ws.yt, 1};
	const int lane = threadIdx.x & 31;
	const uint32_t n = CandCount(nptr, nconst);
	const uint32_t warps = gridDim.x * (blockDim.x / 32);
	unsigned long long ev[3] = {0, 0, 0};
	for (uint32_t k = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; k < n; k += warps) {
		const Cand cd = cands[k];
		double* row = rows + static_cast<long long>(k) * kCols;
		double t[5] = {0, 0, 0, 0, 0}, crlb[5] = {0, 0, 0, 0, 0}, dev = 0;
		RoiAt r;
		if (!Locate(fi, mp, cd, r)) {
			StoreMleRow(row, lane, mp, cd, t, crlb, 0.0, r.ux, r.uy, false);
			continue;
		}
		Pix px = MakePix(mp, r.base, r.W, nullptr, 0);
		ev[2] += InitTheta<MODEL, 32>(mp, px, r, t, xt32, yt32);
		for (int q = lane; q < mp.n; q += 32) {
			const int i = q / mp.roi, j = q - i * mp.roi;
			ws.photons[q] = fmaxf((float(__ldg(r.base + i * r.W + j)) - px.off32) * px.inv32, 0.f);
		}
		__syncwarp();
		Pix ps = px;
		ps.sm = ws.photons;
		ps.ss = 1;
		const float x0 = static_cast<float>(r.x0), y0 = static_cast<float>(r.y0);
		float th[5];
		#pragma unroll
		for (int a = 0; a < 5; ++a) { th[a] = static_cast<float>(t[a]); }
		float G[5], Hm[15];
		float D = Normal<float, MODEL, 32, kFisher>(mp, ps, th, G, Hm, nullptr, xt32, yt32);
		++ev[0];
		bool ok = isfinite(D);
		float lambda = 1e-3f;
		for (int it = 0; ok && it < mp.maxIter; ++it) {
			float rhs[5], dt[5];
			#pragma unroll
			for (int a = 0; a < 5; ++a) { rhs[a] = -G[a]; }
			FixActive32<MODEL>(mp, x0, y0, th, G, Hm, rhs);
			if (!Solve32(Hm, 1.f + lambda, rhs, dt, mp.fallbacks, lane == 0)) {
				lambda *= 10.f;
				if (lambda > 1e7f) { break; }
				continue;
			}
			float tt[5];
			#pragma unroll
			for (int a = 0; a < 5; ++a) { tt[a] = th[a] + dt[a]; }
			Clamp32<MODEL>(mp, x0, y0, tt);
			float Gt[5], Ht[15];
			const float Dt = Normal<float, MODEL, 32, kFisher>(mp, ps, tt, Gt, Ht, nullptr, xt32, yt32);
			++ev[0];
			if (isfinite(Dt) && Dt < D) {
				const bool small = StepSmall(MODEL, th, tt);
				#pragma unroll
				for (int a = 0; a < 5; ++a) { th[a] = tt[a]; G[a] = Gt[a]; }
				#pragma unroll
				for (int a = 0; a < 15; ++a) { Hm[a] = Ht[a]; }
				D = Dt;
				lambda = fmaxf(lambda * 0.1f, 1e-7f);
				if (small) { break; }
			}
			else {
				lambda *= 10.f;
				if (lambda > 1e7f) { break; }
			}
		}
		if (ok) {
			ev[1] += Polish<MODEL, 32>(mp, ps, x0, y0, th, xt32, yt32);
			#pragma unroll
			for (int a = 0; a < 5; ++a) { t[a] = th[a]; }
			ok = Final<MODEL, 32>(mp, px, t, crlb, dev, xt64, yt64);
			++ev[2];
		}
		__syncwarp();  // photons are rewritten for the next candidate
		StoreMleRow(row, lane, mp, cd, t, crlb, dev, r.ux, r.uy, ok);
	}
	if (mp.evals && lane == 0) {
		#pragma unroll
		for (int a = 0; a < 3; ++a) {
			if (ev[a]) { atomicAdd(mp.evals + a, ev[a]); }
		}
	}
}

// ---------------------------------------------------------------------------------------------------------------

int SmCount()
{
	int dev = 0, sms = 148;
	if (cudaGetDevice(&dev) == cudaSuccess) { cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev); }
	return sms;
}

template <typename K>
void AllowSmem(K kernel, size_t bytes)
{
	if (bytes > 48 * 1024) { cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)); }
}

// marks (profiling, or null): 5 events, recorded before the initial values, the LM, the polish, the FP64 pass and
// after it.
template <typename K>
int PersistentBlocks(K kernel, size_t smemBytes, int sms, uint32_t cap)
{
	AllowSmem(kernel, smemBytes);
	int perSm = 0;
	if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, kThreads, smemBytes) != cudaSuccess || perSm < 1) { perSm = 1; }
	return static_cast<int>(std::min<uint32_t>((std::max<uint32_t>(cap, 1) + kThreads - 1) / kThreads, static_cast<uint32_t>(sms * perSm)));
}

// The four-launch pipeline; the LM and polish run with L lanes per ROI (1: a thread per ROI; 2-16: lane groups).
template <int MODEL, int L>
bool LaunchPipeline(const FitImages& fi, const Cand* cands, const uint32_t* nptr, uint32_t nconst,
                    uint32_t cap, const MleParams& mp, double* rows, cudaEvent_t* marks, cudaStream_t st)
{
	const int sms = SmCount();
	const uint32_t blocks = std::min<uint32_t>((std::max<uint32_t>(cap, 1) + kThreads - 1) / kThreads, static_cast<uint32_t>(sms) * 32u);
	const size_t initBytes = static_cast<size_t>(mp.roi) * sizeof(float) * kThreads;
	const size_t slots = L == 1 ? kThreads : kThreads / L;
	const size_t lmBytes = static_cast<size_t>(SlotFloats(mp.n, mp.roi, 3, L)) * sizeof(float) * slots;
	const size_t polishBytes = static_cast<size_t>(SlotFloats(mp.n, mp.roi, 6, L)) * sizeof(float) * slots;
	const size_t finalBytes = static_cast<size_t>(3 * mp.roi) * sizeof(double) * kThreads;
	const uint32_t rois = static_cast<uint32_t>(std::min<unsigned long long>(static_cast<unsigned long long>(cap) * L, 0xffffffffull));
	const int lmBlocks = PersistentBlocks(MleLmKernel<MODEL, L>, lmBytes, sms, rois);
	const int polishBlocks = PersistentBlocks(MlePolishKernel<MODEL, L>, polishBytes, sms, rois);
	if (mp.queue && !PTB_CUDA(cudaMemsetAsync(mp.queue, 0, 2 * sizeof(unsigned int), st))) { return false; }
	if (marks) { cudaEventRecord(marks[0], st); }
	MleInitKernel<MODEL><<<blocks, kThreads, initBytes, st>>>(fi, cands, nptr, nconst, mp, rows);
	if (marks) { cudaEventRecord(marks[1], st); }
	MleLmKernel<MODEL, L><<<lmBlocks, kThreads, lmBytes, st>>>(fi, cands, nptr, nconst, mp, rows);
	if (marks) { cudaEventRecord(marks[2], st); }
	MlePolishKernel<MODEL, L><<<polishBlocks, kThreads, polishBytes, st>>>(fi, cands, nptr, nconst, mp, rows);
	if (marks) { cudaEventRecord(marks[3], st); }
	MleFinalKernel<MODEL><<<blocks, kThreads, finalBytes, st>>>(fi, cands, nptr, nconst, mp, rows);
	if (marks) { cudaEventRecord(marks[4], st); }
	CountLaunch(4);
	return PTB_LAUNCHED();
}

// marks: the single launch is timed as the LM phase (marks 0-1 before it, marks 2-4 after it).
template <int MODEL>
bool LaunchWarpPerRoi(const FitImages& fi, const Cand* cands, const uint32_t* nptr, uint32_t nconst,
                      uint32_t cap, const MleParams& mp, double* rows, cudaEvent_t* marks, cudaStream_t st)
{
	const uint32_t perBlock = kThreads / 32;
	const uint32_t blocks = std::min<uint32_t>((std::max<uint32_t>(cap, 1) + perBlock - 1) / perBlock, static_cast<uint32_t>(SmCount()) * 32u);
	if (marks) {
		cudaEventRecord(marks[0], st);
		cudaEventRecord(marks[1], st);
	}
	MleWarpKernel<MODEL><<<blocks, kThreads, 0, st>>>(fi, cands, nptr, nconst, mp, rows);
	if (marks) {
		cudaEventRecord(marks[2], st);
		cudaEventRecord(marks[3], st);
		cudaEventRecord(marks[4], st);
	}
	CountLaunch();
	return PTB_LAUNCHED();
}

template <int MODEL>
bool LaunchModel(int lanes, const FitImages& fi, const Cand* cands, const uint32_t* nptr,
                 uint32_t nconst, uint32_t cap, const MleParams& mp, double* rows, cudaEvent_t* marks, cudaStream_t st)
{
	switch (lanes) {
		case 1: return LaunchPipeline<MODEL, 1>(fi, cands, nptr, nconst, cap, mp, rows, marks, st);
		case 2: return LaunchPipeline<MODEL, 2>(fi, cands, nptr, nconst, cap, mp, rows, marks, st);
		case 4: return LaunchPipeline<MODEL, 4>(fi, cands, nptr, nconst, cap, mp, rows, marks, st);
		case 8: return LaunchPipeline<MODEL, 8>(fi, cands, nptr, nconst, cap, mp, rows, marks, st);
		case 16: return LaunchPipeline<MODEL, 16>(fi, cands, nptr, nconst, cap, mp, rows, marks, st);
		default: return LaunchWarpPerRoi<MODEL>(fi, cands, nptr, nconst, cap, mp, rows, marks, st);
	}
}

}  // namespace

// lanes: 1 = thread per ROI, 2 / 4 / 8 / 16 = lane groups per ROI in the LM and polish, anything else = warp per ROI
// (one launch). mp.chunk: candidates a lane or group takes from the work queue at a time. marks: profiling events (5)
// or null.
bool LaunchMle(int lanes, const FitImages& fi, const Cand* cands, const uint32_t* nptr, uint32_t nconst,
               uint32_t cap, const MleParams& mp, double* rows, cudaEvent_t* marks, cudaStream_t st)
{
	if (mp.roi < 1 || mp.roi > kMaxRoi) {
		SetError("MLE fit: ROI size must be 1-15");
		return false;
	}
	switch (mp.model) {
		case 6: return LaunchModel<6>(lanes, fi, cands, nptr, nconst, cap, mp, rows, marks, st);
		case 7: return LaunchModel<7>(lanes, fi, cands, nptr, nconst, cap, mp, rows, marks, st);
		case 8: return LaunchModel<8>(lanes, fi, cands, nptr, nconst, cap, mp, rows, marks, st);
		default: return false;
	}
}

}  // namespace ptb
