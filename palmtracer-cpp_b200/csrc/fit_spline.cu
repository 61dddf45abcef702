// Cubic-spline PSF fit, EMCCD Poisson deviance (mode 5), one warp per ROI, FP64.
//
// Reference: lib/fit/SplineFit.cpp:53-318 with the bounds of lib/fit/Fitting.cpp:161-172, the centre of mass of
// lib/signal_processing/Matrix.cpp:245-269, its Cholesky (:272-294) and LU inverse (:358-410). Every behaviour of
// the reference is kept, including the ones that look accidental: the deviance accumulator starts at DBL_MAX and
// is never reset (so updates are always accepted and the loop stops after the third iteration unless the deviance
// turns NaN), the ROI row index drives the spline's x cell and the column index its y cell, and the output columns
// carry CRLB values (Offset = CRLB(bg), Intensity/Amplitude = CRLB(A), QualityXY = mean CRLB(x, y), QualityZ =
// deltaZ * CRLB(z)).
//
// The coefficient table is stored cell-major on the device ([cell][64], transposed from the reference's [64][cell])
// so that the 64 coefficients one pixel needs are one contiguous 512-byte run.
#include <algorithm>

#include "pt_common.cuh"

namespace ptb {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarps = 4;

__device__ __forceinline__ double WarpSumD(double v)
{
	#pragma unroll
	for (int d = 16; d > 0; d >>= 1) { v += __shfl_xor_sync(kFull, v, d); }
	return v;
}

struct Patch {
	double f[64], dx[64], dy[64], dz[64];
};

// Monomial weights x^k y^j z^i and their derivatives (SplineFit.cpp:296-318), two entries per lane.
__device__ void PatchWeights(Patch& P, double x, double y, double z)
{
	const int lane = threadIdx.x & 31;
	for (int id = lane; id < 64; id += 32) {
		const int i = id >> 4, j = (id >> 2) & 3, k = id & 3;
		double cz = 1.0, cy = 1.0, cx = 1.0, cxm = 1.0;
		for (int a = 0; a < i; ++a) { cz *= z; }
		for (int a = 0; a < j; ++a) { cy *= y; }
		for (int a = 0; a < k; ++a) { cxm = cx; cx *= x; }
		const double zy = cz * cy;
		P.f[id] = zy * cx;
		P.dx[id] = k > 0 ? static_cast<double>(k) * (zy * cxm) : 0.0;
		// derivative in y: j * x^k y^(j-1) z^i; in z: i * x^k y^j z^(i-1)
		double cym = 1.0, czm = 1.0;
		for (int a = 0; a + 1 < j; ++a) { cym *= y; }
		for (int a = 0; a + 1 < i; ++a) { czm *= z; }
		P.dy[id] = j > 0 ? static_cast<double>(j) * (cz * cym * cx) : 0.0;
		P.dz[id] = i > 0 ? static_cast<double>(i) * (czm * cy * cx) : 0.0;
	}
	__syncwarp();
}

// size_t semantics of Vec3I::Clamp: a negative index wraps and clamps to the upper bound.
__device__ __forceinline__ long long ClampCell(long long v, int dim) { return (v < 0 || v > dim - 1) ? dim - 1 : v; }

// Model and derivatives at one ROI pixel (SplineFit.cpp:219-240).
__device__ __forceinline__ double Eval(const FitParams& fp, const Patch& P, long long cx, long long cy, long long cz,
                                       const double* p, double dudt[5])
{
	const long long x = ClampCell(cx, fp.sx), y = ClampCell(cy, fp.sy), z = ClampCell(cz, fp.sz);
	const double* c = fp.coeffs + (((z * fp.sy) + y) * fp.sx + x) * 64;
	double s1 = 0, s2 = 0, s3 = 0, s4 = 0;
	#pragma unroll 8
	for (int i = 0; i < 64; ++i) {
		const double v = __ldg(c + i);
		s1 += P.f[i] * v;
		s2 += P.dx[i] * v;
		s3 += P.dy[i] * v;
		s4 += P.dz[i] * v;
	}
	dudt[0] = 1;
	dudt[1] = s1;
	dudt[2] = s2 * (-1 * p[1]);
	dudt[3] = s3 * (-1 * p[1]);
	dudt[4] = s4 * p[1];
	return p[0] + (p[1] * dudt[1]);
}

__device__ void StoreRow(double* row, double segI, double surf, double x, double y, double z, double off, double amp,
                         double qxy, double qz, bool sentinel)
{
	const int lane = threadIdx.x & 31;
	double v[kCols];
	v[cId] = 0; v[cPlane] = 0; v[cIndex] = 0; v[cChannel] = -1;
	v[cX] = x; v[cY] = y; v[cZ] = z;
	v[cIntensity] = amp;
	v[cSigmaX] = sentinel ? -1 : 0; v[cSigmaY] = sentinel ? -1 : 0; v[cTheta] = sentinel ? -1 : 0;
	v[cQualityXY] = qxy; v[cQualityZ] = qz;
	v[cAmplitude] = amp; v[cOffset] = off;
	v[cSegIntensity] = segI; v[cSurface] = surf;
	v[cCircularity] = 1.0;
	#pragma unroll
	for (int c = 0; c < kCols; ++c) {
		if (lane == c) { row[c] = v[c]; }
	}
}

__global__ void __launch_bounds__(32 * kWarps) SplineFitKernel(const uint16_t* __restrict__ img, int H, int W, long long N,
                                                                const Cand* __restrict__ cands, const uint32_t* nptr,
                                                                uint32_t nconst, FitParams fp, double* rows)
{
	__shared__ Patch patches[kWarps];
	Patch& P = patches[threadIdx.x >> 5];
	const int lane = threadIdx.x & 31;
	const uint32_t n = nptr ? *nptr : nconst;
	const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
	const int roi = fp.roi, hh = fp.half, npx = fp.n;
	for (uint32_t k = warp; k < n; k += nw) {
		const Cand cd = cands[k];
		double* row = rows + static_cast<long long>(k) * kCols;
		const bool nonneg = cd.x >= 0.0 && cd.y >= 0.0;
		const unsigned long long ux = nonneg ? static_cast<unsigned long long>(cd.x) : 0ull;
		const unsigned long long uy = nonneg ? static_cast<unsigned long long>(cd.y) : 0ull;
		const unsigned long long h = static_cast<unsigned long long>(hh);
		if (!nonneg || h > ux || ux >= static_cast<unsigned long long>(W) - h || h > uy || uy >= static_cast<unsigned long long>(H) - h) {
			StoreRow(row, cd.intensity, cd.surf, cd.x, cd.y, 0, -1, -1, -1, -1, true);
			continue;
		}
		const uint16_t* base = img + static_cast<long long>(cd.frame) * N + static_cast<long long>(uy - h) * W + static_cast<long long>(ux - h);
		// ROI min / max and centre of mass (rows weight y, columns weight x)
		double vmin = 1e300, vmax = -1e300, sx = 0, sy = 0, sv = 0;
		for (int idx = lane; idx < npx; idx += 32) {
			const int i = idx / roi, j = idx - i * roi;
			const double v = static_cast<double>(__ldg(base + static_cast<long long>(i) * W + j));
			vmin = fmin(vmin, v);
			vmax = fmax(vmax, v);
			sy += v * static_cast<double>(i);
			sx += v * static_cast<double>(j);
			sv += v;
		}
		#pragma unroll
		for (int d = 16; d > 0; d >>= 1) {
			vmin = fmin(vmin, __shfl_xor_sync(kFull, vmin, d));
			vmax = fmax(vmax, __shfl_xor_sync(kFull, vmax, d));
		}
		sx = WarpSumD(sx);
		sy = WarpSumD(sy);
		sv = WarpSumD(sv);
		double x0, y0;
		if (sv > 0) { x0 = sx / sv; y0 = sy / sv; }
		else { x0 = static_cast<double>(roi) / 2.0; y0 = static_cast<double>(roi) / 2.0; }
		const double roiC = (fp.roiParam - 1) / 2.0, roiD = fp.roiParam / 4.0;
		const double lo[5] = {-0.01, -1, roiC - roiD, roiC - roiD, 0};
		const double hi[5] = {0.01, 1, roiC + roiD, roiC + roiD, static_cast<double>(fp.sz)};
		double p[5] = {vmin, (vmax - vmin) * fp.intensityRatio, x0, y0, fp.initZ};
		#pragma unroll
		for (int a = 0; a < 5; ++a) { p[a] = fmin(fmax(p[a], lo[a]), hi[a]); }
		double jump[5] = {fmax(20.0, p[1]), fmax(100.0, p[1]), 1.0, 1.0, fmax(static_cast<double>(fp.sz) / 3.0, 2.0)};
		double lambda = 0.1, err = 1.7976931348623157e308, mu = 1 + lambda;
		double upd[5] = {0, 0, 0, 0, 0};
		auto cell = [&](const double* pp, long long& xi, long long& yi, long long& zi) {
			const double xr = -1 * (pp[2] - static_cast<double>(hh) + 0.5), yr = -1 * (pp[3] - static_cast<double>(hh) + 0.5);
			xi = static_cast<int>(floor(xr));
			yi = static_cast<int>(floor(yr));
			zi = static_cast<int>(floor(pp[4]));
			PatchWeights(P, xr - static_cast<double>(xi), yr - static_cast<double>(yi), pp[4] - static_cast<double>(zi));
		};
		bool stop = false;
		int it = 0;
		while (!stop) {
			++it;
			const double oldErr = err, oldLambda = lambda;
			double oldP[5], oldUpd[5];
			#pragma unroll
			for (int a = 0; a < 5; ++a) { oldP[a] = p[a]; oldUpd[a] = upd[a]; upd[a] = 0; }
			long long xi, yi, zi;
			cell(p, xi, yi, zi);
			double dev = 0, jac[5] = {0, 0, 0, 0, 0}, hs[15] = {};
			for (int idx = lane; idx < npx; idx += 32) {
				const int i = idx / roi, j = idx - i * roi;
				const double d = static_cast<double>(__ldg(base + static_cast<long long>(i) * W + j));
				double dudt[5];
				const double model = Eval(fp, P, xi + i + fp.offsetXY, yi + j + fp.offsetXY, zi, p, dudt);
				dev += d > 0 ? 2 * (model - d - (d * log(model / d))) : 2 * model;
				const double t1 = 1 - (d / model), t2 = d / (model * model);
				int q = 0;
				#pragma unroll
				for (int a = 0; a < 5; ++a) {
					jac[a] += t1 * dudt[a];
					#pragma unroll
					for (int b = a; b < 5; ++b) { hs[q++] += t2 * dudt[a] * dudt[b]; }
				}
			}
			err = err + WarpSumD(dev);
			double hess[5][5];
			{
				int q = 0;
				#pragma unroll
				for (int a = 0; a < 5; ++a) {
					jac[a] = WarpSumD(jac[a]);
					#pragma unroll
					for (int b = a; b < 5; ++b) {
						hess[a][b] = WarpSumD(hs[q++]);
						hess[b][a] = hess[a][b];
					}
				}
			}
			#pragma unroll
			for (int a = 0; a < 5; ++a) { hess[a][a] = hess[a][a] * mu; }
			// Cholesky, lower factor u (Matrix.cpp:272-294)
			double u[5][5] = {};
			bool chol = true;
			#pragma unroll
			for (int a = 0; a < 5; ++a) {
				#pragma unroll
				for (int b = 0; b <= a; ++b) {
					double s = 0;
					#pragma unroll
					for (int c = 0; c < b; ++c) { s += u[a][c] * u[b][c]; }
					if (a == b) {
						if (hess[a][a] - s >= 0) { u[a][b] = sqrt(hess[a][a] - s); }
						else { chol = false; }
					}
					else { u[a][b] = 1.0 / u[b][b] * (hess[a][b] - s); }
				}
			}
			if (chol) {
				double yv[5];
				#pragma unroll
				for (int a = 0; a < 5; ++a) {
					yv[a] = jac[a];
					#pragma unroll
					for (int b = 0; b < a; ++b) { yv[a] -= u[a][b] * yv[b]; }
					yv[a] /= u[a][a];
				}
				#pragma unroll
				for (int a = 4; a >= 0; --a) {
					upd[a] = yv[a];
					#pragma unroll
					for (int b = a + 1; b < 5; ++b) { upd[a] -= u[b][a] * upd[b]; }
					upd[a] /= u[a][a];
				}
				#pragma unroll
				for (int a = 0; a < 5; ++a) {
					if (fabs(oldUpd[a]) > kEps && upd[a] / oldUpd[a] < -0.5) { jump[a] *= 0.5; }
					const double scale = upd[a] / (1.0 + (fabs(upd[a]) / jump[a]));
					p[a] -= scale;
					p[a] = fmin(fmax(p[a], lo[a]), hi[a]);
					upd[a] = scale;
				}
			}
			if (!chol || err > oldErr) {
				err = oldErr;
				#pragma unroll
				for (int a = 0; a < 5; ++a) { p[a] = oldP[a]; upd[a] = oldUpd[a]; }
				lambda = oldLambda;
				mu = fmax((1 + (lambda * 10)) / (1 + lambda), 1.3);
				lambda = 10 * lambda;
			}
			else {
				lambda = 0.1 * lambda;
				mu = 1 + lambda;
			}
			if (it >= kMaxIter) { stop = true; }
			if (it > 2 && (err < 1e-6 || fabs(err - oldErr) / err < 1e-6)) { stop = true; }
		}
		// CRLB from the Fisher information at the final parameters (SplineFit.cpp:164-205)
		long long xi, yi, zi;
		cell(p, xi, yi, zi);
		double fs[15] = {};
		for (int idx = lane; idx < npx; idx += 32) {
			const int i = idx / roi, j = idx - i * roi;
			double dudt[5];
			const double model = Eval(fp, P, xi + i + fp.offsetXY, yi + j + fp.offsetXY, zi, p, dudt);
			int q = 0;
			#pragma unroll
			for (int a = 0; a < 5; ++a) {
				#pragma unroll
				for (int b = a; b < 5; ++b) { fs[q++] += dudt[b] * dudt[a] / model; }
			}
		}
		double m[25];
		{
			int q = 0;
			#pragma unroll
			for (int a = 0; a < 5; ++a) {
				#pragma unroll
				for (int b = a; b < 5; ++b) {
					const double v = WarpSumD(fs[q++]);
					m[a * 5 + b] = v;
					m[b * 5 + a] = v;
				}
			}
		}
		#pragma unroll
		for (int a = 0; a < 5; ++a) {
			if (fabs(m[a * 5 + a]) < 2.220446049250313e-16) { m[a * 5 + a] = 1e-10; }
		}
		// LU inverse without pivoting, column-major as Matrix.cpp:358-410 (only the diagonal of the inverse is kept)
		double crlb[5];
		{
			double acc = 0;
			#pragma unroll
			for (int j = 0; j < 5; ++j) {
				#pragma unroll
				for (int i = 1; i <= j; ++i) {
					#pragma unroll
					for (int q = 0; q <= i - 1; ++q) { acc += m[i + q * 5] * m[q + j * 5]; }
					m[i + j * 5] -= acc;
					acc = 0;
				}
				#pragma unroll
				for (int i = j + 1; i < 5; ++i) {
					if (j > 0) {
						#pragma unroll
						for (int q = 0; q <= j - 1; ++q) { acc += m[i + q * 5] * m[q + j * 5]; }
						m[i + j * 5] = (1 / m[j + j * 5]) * (m[i + j * 5] - acc);
						acc = 0;
					}
					else { m[i + j * 5] = (1 / m[j + j * 5]) * m[i + j * 5]; }
				}
			}
			#pragma unroll
			for (int num = 0; num < 5; ++num) {
				double yv[5], out[5];
				yv[0] = num == 0 ? 1 : 0;
				#pragma unroll
				for (int i = 1; i < 5; ++i) {
					#pragma unroll
					for (int j = 0; j <= i - 1; ++j) { acc += m[i + j * 5] * yv[j]; }
					yv[i] = (i == num ? 1.0 : 0.0) - acc;
					acc = 0;
				}
				out[4] = yv[4] / m[4 + 4 * 5];
				#pragma unroll
				for (int i = 3; i >= 0; --i) {
					#pragma unroll
					for (int j = i + 1; j < 5; ++j) { acc += m[i + j * 5] * out[j]; }
					out[i] = (1 / m[i + i * 5]) * (yv[i] - acc);
					acc = 0;
				}
				const double v = out[num];
				crlb[num] = isnan(v) ? v : (v >= 0 ? sqrt(v) : 0.0);  // real part of the complex square root
			}
		}
		const double xo = p[2] - static_cast<double>(hh) + cd.x;
		const double yo = p[3] - static_cast<double>(hh) + cd.y;
		const double zo = fp.deltaZ * (p[4] - fp.initZ);
		StoreRow(row, cd.intensity, cd.surf, xo, yo, zo, crlb[0], crlb[1], (crlb[2] + crlb[3]) / 2, fp.deltaZ * crlb[4], false);
	}
}

}  // namespace

bool LaunchSpline(const uint16_t* img, int H, int W, long long N, const Cand* cands, const uint32_t* nptr, uint32_t nconst,
                  uint32_t cap, const FitParams& fp, double* rows, cudaStream_t st)
{
	const uint32_t blocks = std::min<uint32_t>((std::max<uint32_t>(cap, 1) + kWarps - 1) / kWarps, 148u * 16u);
	SplineFitKernel<<<blocks, 32 * kWarps, 0, st>>>(img, H, W, N, cands, nptr, nconst, fp, rows);
	CountLaunch();
	return PTB_LAUNCHED();
}

}  // namespace ptb
