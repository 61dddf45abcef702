// Poisson maximum-likelihood fits (modes 6 Gaussian, 7 astigmatic 3D, 8 cubic-spline 3D) of (bg, I, x, y, s),
// s = sigma (mode 6), z in nm (mode 7) or the spline's z coordinate (mode 8). No counterpart in the reference; the
// model maths, the algorithm and the FP64 oracle are in oracle/pt_oracle.cpp (MleFit), which this file follows step
// for step: initial values, bounds, FP64 axial pre-scan, damped Fisher-scoring LM on the Poisson deviance, undamped
// FP64 Fisher steps to a 1e-10 relative step and the CRLB from the FP64 Fisher information.
//
// Precision: the LM iterations run in FP32. The 5x5 damped system is factored by an FP32 Cholesky; when a pivot is not
// positive or the pivot ratio min(L_ii^2) / max(A_ii) falls below 1e-5 the same system is re-factored in FP64. The
// final polish, the log-likelihood (deviance) and the CRLB are computed in FP64.
//
// Mapping: L lanes per ROI (L = 1, 8, 16 or 32; 32 / L ROIs per warp), chosen by the autotuner in engine.cu. Sums over
// pixels are reduced with shuffles masked to the ROI's lane group. For modes 6 and 7 the pixel-integrated Gaussian is
// separable, so each iteration evaluates the erf terms once per ROI column and row into a per-group shared table.
// For mode 8 the monomial weights are the same for every pixel of the ROI (pixels differ by whole cells), so each
// lane forms them once per iteration; the table is FP32, cell-major ([cell][64]).
#include <algorithm>

#include "pt_common.cuh"

namespace ptb {

namespace {

constexpr int kMaxRoi = 15;
constexpr int kThreads = 64;

template <typename T> __device__ __forceinline__ T Erf(T x);
template <> __device__ __forceinline__ float Erf<float>(float x) { return erff(x); }
template <> __device__ __forceinline__ double Erf<double>(double x) { return erf(x); }
template <typename T> __device__ __forceinline__ T Ex(T x);
template <> __device__ __forceinline__ float Ex<float>(float x) { return expf(x); }
template <> __device__ __forceinline__ double Ex<double>(double x) { return exp(x); }
template <typename T> __device__ __forceinline__ T Ln(T x);
template <> __device__ __forceinline__ float Ln<float>(float x) { return logf(x); }
template <> __device__ __forceinline__ double Ln<double>(double x) { return log(x); }

template <int L, typename T>
__device__ __forceinline__ T GroupSum(T v, unsigned mask)
{
	#pragma unroll
	for (int d = L / 2; d > 0; d >>= 1) { v += __shfl_xor_sync(mask, v, d); }
	return v;
}

template <typename T>
__device__ __forceinline__ void Erf1D(T c, T x, T s, T& e, T& dx, T& ds)
{
	const T k = T(1) / (T(1.4142135623730951) * s);
	const T a = (c - x - T(0.5)) * k, b = (c - x + T(0.5)) * k;
	const T ea = Ex<T>(-a * a), eb = Ex<T>(-b * b);
	e = T(0.5) * (Erf<T>(b) - Erf<T>(a));
	dx = (ea - eb) / (T(2.5066282746310002) * s);
	ds = (a * ea - b * eb) / (T(1.7724538509055160) * s);
}

template <typename T>
__device__ __forceinline__ void AstigSigma(const double* m, double pixelSize, T z, T& s, T& ds)
{
	const T u = (z - T(m[0])) / T(m[1]);
	const T poly = T(1) + u * u + T(m[2]) * u * u * u + T(m[3]) * u * u * u * u;
	const T k = T(m[4] / pixelSize);
	if (poly <= T(1e-12)) { s = k * T(1e-6); ds = T(0); return; }
	const T r = sqrt(poly);
	s = k * r;
	ds = k * (T(2) * u + T(3 * m[2]) * u * u + T(4 * m[3]) * u * u * u) / (T(2) * r * T(m[1]));
}

struct Group {
	int gl;          // lane within the ROI group
	unsigned mask;   // lanes of the group
	void* tab;       // per-group shared scratch (erf tables)
};

// Deviance D and (when FULL) gradient G and Fisher-scoring matrix H (upper triangle, 15 entries) at theta.
template <typename T, int MODEL, int L, bool FULL>
__device__ T Normal(const MleParams& mp, const uint16_t* roiBase, int W, const T th[5], T G[5], T Hm[15], const Group& grp)
{
	const int roi = mp.roi, h = mp.half, n = mp.n;
	T* tab = static_cast<T*>(grp.tab);  // [6][kMaxRoi]: ex, edx, eds, ey, edy, eds_y
	T sx = th[4], sy = th[4], dsx = T(1), dsy = T(1);
	if constexpr (MODEL == 7) {
		AstigSigma<T>(mp.astig, mp.pixelSize, th[4], sx, dsx);
		AstigSigma<T>(mp.astig + 5, mp.pixelSize, th[4], sy, dsy);
	}
	T px[4], py[4], pz[4], dpx[4], dpy[4], dpz[4];
	int ix0 = 0, iy0 = 0, iz = 0;
	if constexpr (MODEL == 6 || MODEL == 7) {
		for (int k = grp.gl; k < roi; k += L) {
			T e, dx, ds;
			Erf1D<T>(T(k - h), th[2], sx, e, dx, ds);
			tab[0 * kMaxRoi + k] = e;
			tab[1 * kMaxRoi + k] = dx;
			tab[2 * kMaxRoi + k] = ds;
			Erf1D<T>(T(k - h), th[3], sy, e, dx, ds);
			tab[3 * kMaxRoi + k] = e;
			tab[4 * kMaxRoi + k] = dx;
			tab[5 * kMaxRoi + k] = ds;
		}
		__syncwarp(grp.mask);
	}
	else {
		// cell of ROI pixel (0, 0) and the common fractional offsets
		const T X = T((mp.sx - 1) * 0.5) - T(h) - th[2], Y = T((mp.sy - 1) * 0.5) - T(h) - th[3];
		const T fxi = floor(X), fyi = floor(Y), fzi = floor(th[4]);
		ix0 = static_cast<int>(fxi);
		iy0 = static_cast<int>(fyi);
		iz = min(max(static_cast<int>(fzi), 0), mp.sz - 1);
		const T fx = X - fxi, fy = Y - fyi, fz = th[4] - T(iz);
		px[0] = T(1); px[1] = fx; px[2] = fx * fx; px[3] = fx * fx * fx;
		py[0] = T(1); py[1] = fy; py[2] = fy * fy; py[3] = fy * fy * fy;
		pz[0] = T(1); pz[1] = fz; pz[2] = fz * fz; pz[3] = fz * fz * fz;
		dpx[0] = T(0); dpx[1] = T(1); dpx[2] = T(2) * fx; dpx[3] = T(3) * fx * fx;
		dpy[0] = T(0); dpy[1] = T(1); dpy[2] = T(2) * fy; dpy[3] = T(3) * fy * fy;
		dpz[0] = T(0); dpz[1] = T(1); dpz[2] = T(2) * fz; dpz[3] = T(3) * fz * fz;
	}
	T D = T(0);
	if constexpr (FULL) {
		#pragma unroll
		for (int a = 0; a < 5; ++a) { G[a] = T(0); }
		#pragma unroll
		for (int a = 0; a < 15; ++a) { Hm[a] = T(0); }
	}
	const T offset = T(mp.offset), invGain = T(1.0 / mp.gain);
	int i = grp.gl / roi, j = grp.gl - i * roi;
	for (int idx = grp.gl; idx < n; idx += L) {
		const T adu = T(__ldg(roiBase + static_cast<long long>(i) * W + j));
		const T d = max((adu - offset) * invGain, T(0));
		T psf, g2, g3, g4;
		if constexpr (MODEL == 6 || MODEL == 7) {
			const T ex = tab[j], edx = tab[kMaxRoi + j], esx = tab[2 * kMaxRoi + j];
			const T ey = tab[3 * kMaxRoi + i], edy = tab[4 * kMaxRoi + i], esy = tab[5 * kMaxRoi + i];
			psf = ex * ey;
			g2 = th[1] * edx * ey;
			g3 = th[1] * ex * edy;
			g4 = th[1] * (esx * dsx * ey + ex * esy * dsy);
		}
		else {
			const int cx = min(max(ix0 + j, 0), mp.sx - 1), cy = min(max(iy0 + i, 0), mp.sy - 1);
			const float4* c4 = reinterpret_cast<const float4*>(mp.table + ((static_cast<long long>(iz) * mp.sy + cy) * mp.sx + cx) * 64);
			T v = T(0), vx = T(0), vy = T(0), vz = T(0);
			#pragma unroll
			for (int q = 0; q < 16; ++q) {  // q = zi * 4 + yj: the four x-monomials of one (z, y) pair
				const float4 c = __ldg(c4 + q);
				const int zi = q >> 2, yj = q & 3;
				const T w = pz[zi] * py[yj];
				const T sxv = T(c.x) * px[0] + T(c.y) * px[1] + T(c.z) * px[2] + T(c.w) * px[3];
				const T sdx = T(c.y) * dpx[1] + T(c.z) * dpx[2] + T(c.w) * dpx[3];
				v += w * sxv;
				vx += w * sdx;
				vy += pz[zi] * dpy[yj] * sxv;
				vz += dpz[zi] * py[yj] * sxv;
			}
			psf = v;
			g2 = -th[1] * vx;
			g3 = -th[1] * vy;
			g4 = th[1] * vz;
		}
		const T mu = max(th[0] + th[1] * psf, T(1e-6));
		D += d > T(0) ? T(2) * (mu - d - d * Ln<T>(mu / d)) : T(2) * mu;
		if constexpr (FULL) {
			const T gk[5] = {T(1), psf, g2, g3, g4};
			const T w1 = T(2) * (T(1) - d / mu), w2 = T(2) / mu;
			int q = 0;
			#pragma unroll
			for (int a = 0; a < 5; ++a) {
				G[a] += w1 * gk[a];
				const T wa = w2 * gk[a];
				#pragma unroll
				for (int b = a; b < 5; ++b) { Hm[q++] += wa * gk[b]; }
			}
		}
		j += L;
		while (j >= roi) { j -= roi; ++i; }
	}
	if constexpr (MODEL == 6 || MODEL == 7) { __syncwarp(grp.mask); }  // tables are rewritten by the next call
	D = GroupSum<L>(D, grp.mask);
	if constexpr (FULL) {
		#pragma unroll
		for (int a = 0; a < 5; ++a) { G[a] = GroupSum<L>(G[a], grp.mask); }
		#pragma unroll
		for (int a = 0; a < 15; ++a) { Hm[a] = GroupSum<L>(Hm[a], grp.mask); }
	}
	return D;
}

__device__ __forceinline__ int Ut(int a, int b) { return a <= b ? a * 5 - (a * (a - 1)) / 2 + (b - a) : b * 5 - (b * (b - 1)) / 2 + (a - b); }

// Cholesky solve of the packed symmetric system (upper triangle) with the given diagonal scaling.
template <typename T>
__device__ bool Chol5(const T Hm[15], T diagScale, const T rhs[5], T x[5], T* pivotRatio)
{
	T Lm[5][5];
	T maxDiag = T(0), minPiv = T(3e38);
	#pragma unroll
	for (int i = 0; i < 5; ++i) {
		#pragma unroll
		for (int j = 0; j <= i; ++j) {
			T s = Hm[Ut(i, j)];
			if (i == j) { s *= diagScale; maxDiag = max(maxDiag, s); }
			#pragma unroll
			for (int k = 0; k < j; ++k) { s -= Lm[i][k] * Lm[j][k]; }
			if (i == j) {
				if (!(s > T(0))) { return false; }
				minPiv = min(minPiv, s);
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
	if (pivotRatio) { *pivotRatio = maxDiag > T(0) ? minPiv / maxDiag : T(0); }
	return true;
}

__device__ void StoreMleRow(double* row, int lane, const MleParams& mp, const Cand& cd, const double t[5], const double crlb[5],
                            unsigned long long ux, unsigned long long uy, bool ok)
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
			AstigSigma<double>(mp.astig, mp.pixelSize, t[4], sx, d1);
			AstigSigma<double>(mp.astig + 5, mp.pixelSize, t[4], sy, d2);
			z = t[4];
			qz = crlb[4];
		}
		if (mp.model == 8) { sx = sy = 0; z = mp.dz * (t[4] - mp.sz / 2.0); qz = mp.dz * crlb[4]; }
		v[cX] = static_cast<double>(ux) + t[2];
		v[cY] = static_cast<double>(uy) + t[3];
		v[cZ] = z;
		v[cIntensity] = t[1];
		v[cSigmaX] = sx; v[cSigmaY] = sy; v[cTheta] = 0;
		v[cQualityXY] = qxy; v[cQualityZ] = qz;
		v[cAmplitude] = (sx > 0 && sy > 0) ? t[1] / (6.283185307179586 * sx * sy) : t[1];
		v[cOffset] = t[0];
		v[cCircularity] = (sx > kEps && sy > kEps) ? fmin(sx, sy) / fmax(sx, sy) : 1;
	}
	v[cSegIntensity] = cd.intensity; v[cSurface] = cd.surf;
	#pragma unroll
	for (int c = 0; c < kCols; ++c) {
		if (lane == c) { row[c] = v[c]; }
	}
}

template <int MODEL, int L>
__global__ void __launch_bounds__(kThreads) MleKernel(const uint16_t* __restrict__ img, int H, int W, long long N,
                                                      const Cand* __restrict__ cands, const uint32_t* nptr, uint32_t nconst,
                                                      MleParams mp, double* rows)
{
	constexpr int kGroups = kThreads / L;
	__shared__ double scratch[kGroups][6 * kMaxRoi];
	const int lane = threadIdx.x & 31;
	const int gIdx = threadIdx.x / L;
	Group grp;
	grp.gl = threadIdx.x % L;
	grp.mask = L == 32 ? 0xffffffffu : (((1u << L) - 1u) << ((lane / L) * L));
	grp.tab = scratch[gIdx];
	const uint32_t n = nptr ? *nptr : nconst;
	const uint32_t first = (blockIdx.x * blockDim.x + threadIdx.x) / L;
	const uint32_t stride = (gridDim.x * blockDim.x) / L;
	for (uint32_t k = first; k < n; k += stride) {
		const Cand cd = cands[k];
		double* row = rows + static_cast<long long>(k) * kCols;
		const bool nonneg = cd.x >= 0.0 && cd.y >= 0.0;
		const unsigned long long ux = nonneg ? static_cast<unsigned long long>(cd.x) : 0ull;
		const unsigned long long uy = nonneg ? static_cast<unsigned long long>(cd.y) : 0ull;
		const unsigned long long hh = static_cast<unsigned long long>(mp.half);
		double t[5] = {0, 0, 0, 0, 0}, crlb[5] = {0, 0, 0, 0, 0};
		const int rowLane = L == 32 ? lane : grp.gl;  // lanes of the group write the row columns
		if (!nonneg || hh > ux || ux >= static_cast<unsigned long long>(W) - hh || hh > uy || uy >= static_cast<unsigned long long>(H) - hh) {
			if (L >= kCols) { StoreMleRow(row, rowLane, mp, cd, t, crlb, ux, uy, false); }
			else if (grp.gl == 0) { for (int c = 0; c < kCols; ++c) { StoreMleRow(row, c, mp, cd, t, crlb, ux, uy, false); } }
			continue;
		}
		const uint16_t* base = img + static_cast<long long>(cd.frame) * N + static_cast<long long>(uy - hh) * W + static_cast<long long>(ux - hh);
		// initial values (MleFit in the oracle): bg = min photons, I = photons above it, x, y = centroid
		float dmin = 3e38f, dsum = 0.f;
		for (int idx = grp.gl; idx < mp.n; idx += L) {
			const int i = idx / mp.roi, j = idx - i * mp.roi;
			const float d = fmaxf((float(__ldg(base + static_cast<long long>(i) * W + j)) - float(mp.offset)) * float(1.0 / mp.gain), 0.f);
			dmin = fminf(dmin, d);
			dsum += d;
		}
		#pragma unroll
		for (int d = L / 2; d > 0; d >>= 1) {
			dmin = fminf(dmin, __shfl_xor_sync(grp.mask, dmin, d));
			dsum += __shfl_xor_sync(grp.mask, dsum, d);
		}
		const double x0 = cd.x - static_cast<double>(ux), y0 = cd.y - static_cast<double>(uy);
		double lo[5], hi[5];
		const double hf = static_cast<double>(mp.half);
		lo[0] = 1e-3; hi[0] = 1e6; lo[1] = 1.0; hi[1] = 1e9;
		lo[2] = fmax(x0 - 2.0, -hf); hi[2] = fmin(x0 + 2.0, hf);
		lo[3] = fmax(y0 - 2.0, -hf); hi[3] = fmin(y0 + 2.0, hf);
		if (MODEL == 6) { lo[4] = 0.5; hi[4] = 5.0; }
		else if (MODEL == 7) { lo[4] = mp.zMin; hi[4] = mp.zMax; }
		else { lo[4] = 0.0; hi[4] = static_cast<double>(mp.sz) - 1e-6; }
		float th[5];
		th[0] = fmaxf(dmin, 1e-3f);
		th[1] = fmaxf(dsum - th[0] * float(mp.n), 1.f);
		th[2] = float(x0);
		th[3] = float(y0);
		if (MODEL == 6) { th[4] = float(mp.sigma0); }
		else {
			// axial pre-scan in FP64, as in the oracle, so that both start from the same basin
			const int ns = MODEL == 7 ? 16 : 8;
			double tsd[5] = {double(th[0]), double(th[1]), double(th[2]), double(th[3]), 0.0};
			double best = 1e300, bz = 0.5 * (lo[4] + hi[4]);
			for (int s = 0; s < ns; ++s) {
				tsd[4] = lo[4] + (hi[4] - lo[4]) * (s + 0.5) / ns;
				const double D = Normal<double, MODEL, L, false>(mp, base, W, tsd, nullptr, nullptr, grp);
				if (D < best) { best = D; bz = tsd[4]; }
			}
			th[4] = float(bz);
		}
		#pragma unroll
		for (int a = 0; a < 5; ++a) { th[a] = fminf(fmaxf(th[a], float(lo[a])), float(hi[a])); }
		float G[5], Hm[15];
		float D = Normal<float, MODEL, L, true>(mp, base, W, th, G, Hm, grp);
		bool ok = isfinite(D);
		float lambda = 1e-3f;
		for (int it = 0; ok && it < mp.maxIter; ++it) {
			float rhs[5], dt[5];
			#pragma unroll
			for (int a = 0; a < 5; ++a) { rhs[a] = -G[a]; }
			float ratio = 0.f;
			bool solved = Chol5<float>(Hm, 1.f + lambda, rhs, dt, &ratio);
			if (!solved || ratio < 1e-5f) {
				// FP64 re-factorisation of the same damped system
				double Hd[15], rd[5], xd[5];
				#pragma unroll
				for (int a = 0; a < 15; ++a) { Hd[a] = Hm[a]; }
				#pragma unroll
				for (int a = 0; a < 5; ++a) { rd[a] = rhs[a]; }
				solved = Chol5<double>(Hd, 1.0 + lambda, rd, xd, nullptr);
				if (grp.gl == 0 && mp.fallbacks) { atomicAdd(mp.fallbacks, 1u); }
				#pragma unroll
				for (int a = 0; a < 5; ++a) { dt[a] = float(xd[a]); }
			}
			if (!solved) {
				lambda *= 10.f;
				if (lambda > 1e7f) { break; }
				continue;
			}
			float tt[5];
			#pragma unroll
			for (int a = 0; a < 5; ++a) { tt[a] = fminf(fmaxf(th[a] + dt[a], float(lo[a])), float(hi[a])); }
			float Gt[5], Ht[15];
			const float Dt = Normal<float, MODEL, L, true>(mp, base, W, tt, Gt, Ht, grp);
			if (isfinite(Dt) && Dt < D) {
				const float gainRel = (D - Dt) / (Dt + 1.f);
				#pragma unroll
				for (int a = 0; a < 5; ++a) { th[a] = tt[a]; G[a] = Gt[a]; }
				#pragma unroll
				for (int a = 0; a < 15; ++a) { Hm[a] = Ht[a]; }
				D = Dt;
				lambda = fmaxf(lambda * 0.1f, 1e-7f);
				if (gainRel < 1e-6f) { break; }
			}
			else {
				lambda *= 10.f;
				if (lambda > 1e7f) { break; }
			}
		}
		// FP64: undamped Fisher steps to a 1e-10 relative step (at most 10, halving a step that does not lower the
		// deviance up to three times), then the CRLB
		#pragma unroll
		for (int a = 0; a < 5; ++a) { t[a] = th[a]; }
		double Gd[5], Hd[15];
		double Dd = Normal<double, MODEL, L, true>(mp, base, W, t, Gd, Hd, grp);
		ok = ok && isfinite(Dd);
		for (int it = 0; ok && it < 10; ++it) {
			double rhs[5], dt[5], tt[5];
			#pragma unroll
			for (int a = 0; a < 5; ++a) { rhs[a] = -Gd[a]; }
			if (!Chol5<double>(Hd, 1.0, rhs, dt, nullptr)) { break; }
			bool accepted = false;
			double Gt[5], Ht[15], Dt = 0;
			for (int hv = 0; hv < 4 && !accepted; ++hv) {
				#pragma unroll
				for (int a = 0; a < 5; ++a) { tt[a] = fmin(fmax(t[a] + dt[a], lo[a]), hi[a]); }
				Dt = Normal<double, MODEL, L, true>(mp, base, W, tt, Gt, Ht, grp);
				if (isfinite(Dt) && Dt <= Dd) { accepted = true; }
				else {
					#pragma unroll
					for (int a = 0; a < 5; ++a) { dt[a] *= 0.5; }
				}
			}
			if (!accepted) { break; }
			double step = 0;
			#pragma unroll
			for (int a = 0; a < 5; ++a) { step = fmax(step, fabs(tt[a] - t[a]) / fmax(fabs(t[a]), 1.0)); }
			#pragma unroll
			for (int a = 0; a < 5; ++a) { t[a] = tt[a]; Gd[a] = Gt[a]; }
			#pragma unroll
			for (int a = 0; a < 15; ++a) { Hd[a] = Ht[a]; }
			Dd = Dt;
			if (step < 1e-10) { break; }
		}
		if (ok) {
			double F[15];
			#pragma unroll
			for (int a = 0; a < 15; ++a) { F[a] = 0.5 * Hd[a]; }
			#pragma unroll
			for (int a = 0; a < 5; ++a) {
				double e[5] = {0, 0, 0, 0, 0}, col[5];
				e[a] = 1.0;
				if (!Chol5<double>(F, 1.0, e, col, nullptr)) { ok = false; break; }
				crlb[a] = col[a] > 0 ? sqrt(col[a]) : 0.0;
			}
		}
		#pragma unroll
		for (int a = 0; a < 5; ++a) { ok = ok && isfinite(t[a]); }
		if (L >= kCols) { StoreMleRow(row, rowLane, mp, cd, t, crlb, ux, uy, ok); }
		else if (grp.gl == 0) {
			for (int c = 0; c < kCols; ++c) { StoreMleRow(row, c, mp, cd, t, crlb, ux, uy, ok); }
		}
	}
}

template <int MODEL>
bool LaunchModel(int lanes, const uint16_t* img, int H, int W, long long N, const Cand* cands, const uint32_t* nptr,
                 uint32_t nconst, uint32_t cap, const MleParams& mp, double* rows, cudaStream_t st)
{
	const uint32_t perBlock = kThreads / lanes;
	const uint32_t blocks = std::min<uint32_t>((std::max<uint32_t>(cap, 1) + perBlock - 1) / perBlock, 148u * 32u);
	switch (lanes) {
		case 1: MleKernel<MODEL, 1><<<blocks, kThreads, 0, st>>>(img, H, W, N, cands, nptr, nconst, mp, rows); break;
		case 8: MleKernel<MODEL, 8><<<blocks, kThreads, 0, st>>>(img, H, W, N, cands, nptr, nconst, mp, rows); break;
		case 16: MleKernel<MODEL, 16><<<blocks, kThreads, 0, st>>>(img, H, W, N, cands, nptr, nconst, mp, rows); break;
		default: MleKernel<MODEL, 32><<<blocks, kThreads, 0, st>>>(img, H, W, N, cands, nptr, nconst, mp, rows); break;
	}
	CountLaunch();
	return PTB_LAUNCHED();
}

}  // namespace

bool LaunchMle(int lanes, const uint16_t* img, int H, int W, long long N, const Cand* cands, const uint32_t* nptr, uint32_t nconst,
               uint32_t cap, const MleParams& mp, double* rows, cudaStream_t st)
{
	switch (mp.model) {
		case 6: return LaunchModel<6>(lanes, img, H, W, N, cands, nptr, nconst, cap, mp, rows, st);
		case 7: return LaunchModel<7>(lanes, img, H, W, N, cands, nptr, nconst, cap, mp, rows, st);
		case 8: return LaunchModel<8>(lanes, img, H, W, N, cands, nptr, nconst, cap, mp, rows, st);
		default: return false;
	}
}

}  // namespace ptb
