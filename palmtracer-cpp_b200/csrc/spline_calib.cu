// Spline calibration's coefficient producer: the cubic B-spline coefficient table of a PSF volume, written directly
// in the layout the spline fits read (SoA [64][sz][sy][sx], modes 5 and 8).
//
// Reference: lib/signal_processing/BSpline3D.cpp (BSpline3D::BSpline3D :17-45, built by the calibration at
// lib/signal_processing/Spline.cpp:52 with degree 3 and lambda = {0, 0, 100 / dz}), which produces the table as
// [cell][64]. The same four steps:
//   1. smoothing-spline prefilter per axis: for every pole z of the axis, a causal and an anticausal first-order
//      recursion along each line with mirror initialisation over K0 = ceil(log(eps) / log|z|) terms (the recursive
//      B-spline filter of Unser, Aldroubi & Eden 1991; applyFilter :284-331, symExpFilt :438-449); the real part times
//      the axis gain is kept after the axis. Poles: lambda = 0 -> sqrt3 - 2, gain 6; lambda > 0 -> the two roots with
//      |z| <= 1 of the palindromic quartic z^4 + b z^3 + c z^2 + b z + 1, b = -4 + 1 / (6 lambda),
//      c = 6 + 2 / (3 lambda), gain 1 / lambda (getPolesFilter :197-214; found here in closed form: w = z + 1/z
//      solves w^2 + b w + c - 2 = 0);
//   2. the spline's values at the voxel centres with the volume mirrored by one voxel (interpolate_at at the grid:
//      weights 1/6, 2/3, 1/6 per axis);
//   3./4. those values as cubic B-spline control points, zero outside the volume; per cell the 64 monomial
//      coefficients of that spline (the reference samples it at 1/3 steps and solves the 64 x 64 system; the
//      control-point-to-monomial basis change gives the same polynomial directly).
// Coefficient k = l * 16 + m * 4 + n multiplies zf^l yf^m xf^n of its cell.
#include <cmath>
#include <complex>
#include <vector>

#include "engine.h"

namespace ptb {

namespace {

__device__ __forceinline__ double2 Cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 Cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 Csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

// Mirror index sequence 0, 1, .., n-1, n-2, .., 1, 0, 1, .. entry k (n >= 2).
__device__ __forceinline__ long long Mirror(long long n, long long k)
{
	const long long p = 2 * n - 2;
	const long long m = ((k % p) + p) % p;
	return m < n ? m : p - m;
}

// First element, stride and length of line l along `axis` of a [nz][ny][nx] volume.
__device__ __forceinline__ void Line(long long l, int axis, long long nx, long long ny, long long nz, long long& base, long long& stride,
                                     long long& n)
{
	if (axis == 0) { base = l * nx; stride = 1; n = nx; }
	else if (axis == 1) { base = (l / nx) * nx * ny + l % nx; stride = nx; n = ny; }
	else { base = l; stride = nx * ny; n = nz; }
}

// One thread per line: the symmetric exponential filter of pole z (c0 = -z / (1 - z^2)) in place.
__global__ void FilterLines(double2* v, long long nx, long long ny, long long nz, int axis, double2 z, double2 c0, int k0)
{
	const long long lines = axis == 0 ? ny * nz : (axis == 1 ? nx * nz : nx * ny);
	for (long long l = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; l < lines;
	     l += static_cast<long long>(gridDim.x) * blockDim.x) {
		long long base, stride, n;
		Line(l, axis, nx, ny, nz, base, stride, n);
		double2* x = v + base;
		double2 acc = make_double2(0, 0), zk = make_double2(1, 0);
		for (int k = 0; k < k0; ++k) {
			acc = Cadd(acc, Cmul(zk, x[Mirror(n, k) * stride]));
			zk = Cmul(zk, z);
		}
		const double2 last = x[(n - 1) * stride];
		x[0] = acc;
		double2 prev = acc;
		for (long long k = 1; k < n; ++k) {
			prev = Cadd(x[k * stride], Cmul(z, prev));
			x[k * stride] = prev;
		}
		prev = Cmul(Csub(make_double2(2 * prev.x, 2 * prev.y), last), c0);
		x[(n - 1) * stride] = prev;
		for (long long k = n - 2; k >= 0; --k) {
			prev = Cmul(Csub(prev, x[k * stride]), z);
			x[k * stride] = prev;
		}
	}
}

__global__ void ToComplex(const double* src, double2* dst, long long count)
{
	for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < count; i += static_cast<long long>(gridDim.x) * blockDim.x) {
		dst[i] = make_double2(src[i], 0.0);
	}
}

__global__ void RealTimesGain(double2* v, long long count, double gain)
{
	for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < count; i += static_cast<long long>(gridDim.x) * blockDim.x) {
		v[i] = make_double2(v[i].x * gain, 0.0);
	}
}

// The spline's value at each voxel centre: weights 1/6, 2/3, 1/6 along each axis over the mirrored coefficients.
__global__ void CentreValues(const double2* c, double* out, long long nx, long long ny, long long nz)
{
	const double w[3] = {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0};
	const long long count = nx * ny * nz;
	for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < count; i += static_cast<long long>(gridDim.x) * blockDim.x) {
		const long long x = i % nx, y = (i / nx) % ny, z = i / (nx * ny);
		double r = 0.0;
		for (int a = 0; a < 3; ++a) {
			const long long zz = Mirror(nz, z + a - 1);
			for (int b = 0; b < 3; ++b) {
				const long long yy = Mirror(ny, y + b - 1);
				const double wzy = w[a] * w[b];
				for (int d = 0; d < 3; ++d) { r += wzy * w[d] * c[(zz * ny + yy) * nx + Mirror(nx, x + d - 1)].x; }
			}
		}
		out[i] = r;
	}
}

// Per cell: control points of the cell's 4 x 4 x 4 neighbourhood (zero outside the volume) to the 64 monomial
// coefficients through the cubic B-spline basis in monomial form, one axis at a time; SoA output.
__global__ void CellMonomials(const double* hdr, double* out, long long nx, long long ny, long long nz)
{
	// B-spline segment of control point k - 1 + a over t in [0, 1): sum_p M[a][p] t^p
	const double M[4][4] = {{1.0 / 6, -3.0 / 6, 3.0 / 6, -1.0 / 6}, {4.0 / 6, 0.0, -6.0 / 6, 3.0 / 6},
	                        {1.0 / 6, 3.0 / 6, 3.0 / 6, -3.0 / 6}, {0.0, 0.0, 0.0, 1.0 / 6}};
	const long long cx = nx - 1, cy = ny - 1, cz = nz - 1, cells = cx * cy * cz;
	for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < cells; i += static_cast<long long>(gridDim.x) * blockDim.x) {
		const long long x = i % cx, y = (i / cx) % cy, z = i / (cx * cy);
		double t[4][4][4];  // [z offset][y offset][x power], then [z offset][y power][x power], then powers
		for (int a = 0; a < 4; ++a) {
			const long long zz = z - 1 + a;
			for (int b = 0; b < 4; ++b) {
				const long long yy = y - 1 + b;
				double p[4];
				for (int d = 0; d < 4; ++d) {
					const long long xx = x - 1 + d;
					const bool in = zz >= 0 && zz < nz && yy >= 0 && yy < ny && xx >= 0 && xx < nx;
					p[d] = in ? hdr[(zz * ny + yy) * nx + xx] : 0.0;
				}
				for (int q = 0; q < 4; ++q) { t[a][b][q] = M[0][q] * p[0] + M[1][q] * p[1] + M[2][q] * p[2] + M[3][q] * p[3]; }
			}
			for (int q = 0; q < 4; ++q) {
				double u[4];
				for (int m = 0; m < 4; ++m) { u[m] = M[0][m] * t[a][0][q] + M[1][m] * t[a][1][q] + M[2][m] * t[a][2][q] + M[3][m] * t[a][3][q]; }
				for (int m = 0; m < 4; ++m) { t[a][m][q] = u[m]; }
			}
		}
		for (int m = 0; m < 4; ++m) {
			for (int q = 0; q < 4; ++q) {
				for (int l = 0; l < 4; ++l) {
					const double v = M[0][l] * t[0][m][q] + M[1][l] * t[1][m][q] + M[2][l] * t[2][m][q] + M[3][l] * t[3][m][q];
					out[static_cast<long long>(l * 16 + m * 4 + q) * cells + i] = v;
				}
			}
		}
	}
}

// Poles and gain of the degree-3 smoothing-spline filter for regularisation lambda (see the file comment).
void CubicPoles(double lambda, std::vector<std::complex<double>>& poles, double& gain)
{
	poles.clear();
	if (lambda <= 2.220446049250313e-16) {
		poles.emplace_back(std::sqrt(3.0) - 2.0);
		gain = 6.0;
		return;
	}
	const double b = -4.0 + 1.0 / (6.0 * lambda), c = 6.0 + 2.0 / (3.0 * lambda);
	const std::complex<double> disc = std::sqrt(std::complex<double>(b * b - 4.0 * (c - 2.0), 0.0));
	for (const std::complex<double> w : {(-b + disc) / 2.0, (-b - disc) / 2.0}) {
		const std::complex<double> r = std::sqrt(w * w - 4.0);
		const std::complex<double> z1 = (w - r) / 2.0, z2 = (w + r) / 2.0;
		poles.push_back(std::abs(z1) <= 1.0 ? z1 : z2);
	}
	gain = 1.0 / lambda;
}

}  // namespace

// Host volume [nz][ny][nx] -> host coefficients SoA [64][nz-1][ny-1][nx-1]; lambda per axis (x, y, z) or null.
// Returns false (error recorded) for dimensions below 2 or a failed CUDA call.
bool SplineCoefficients(const double* volume, uint64_t nx, uint64_t ny, uint64_t nz, const double* lambda, double* out, cudaStream_t st)
{
	if (nx < 2 || ny < 2 || nz < 2) {
		SetError("spline calibration: every dimension must be at least 2");
		return false;
	}
	const unsigned long long count = nx * ny * nz;
	const unsigned long long cells = (nx - 1) * (ny - 1) * (nz - 1);
	double2* c = nullptr;
	double* hdr = nullptr;
	double* coef = nullptr;
	bool ok = PTB_CUDA(cudaMallocAsync(&c, count * sizeof(double2), st));
	ok = ok && PTB_CUDA(cudaMallocAsync(&hdr, count * sizeof(double), st));
	ok = ok && PTB_CUDA(cudaMallocAsync(&coef, cells * 64 * sizeof(double), st));
	// complex working copy: real parts from the volume (staged in hdr), imaginary parts zero
	ok = ok && PTB_CUDA(cudaMemcpyAsync(hdr, volume, count * sizeof(double), cudaMemcpyHostToDevice, st));
	const int threads = 128, grid = 148 * 8;
	const long long dims[3] = {static_cast<long long>(nx), static_cast<long long>(ny), static_cast<long long>(nz)};
	if (ok) {
		ToComplex<<<grid, threads, 0, st>>>(hdr, c, static_cast<long long>(count));
		CountLaunch();
		ok = PTB_LAUNCHED();
	}
	for (int axis = 0; axis < 3 && ok; ++axis) {
		std::vector<std::complex<double>> poles;
		double gain = 1.0;
		CubicPoles(lambda ? lambda[axis] : 0.0, poles, gain);
		for (const std::complex<double>& z : poles) {
			const std::complex<double> c0 = -z / (1.0 - z * z);
			const int k0 = static_cast<int>(std::ceil(std::log(2.220446049250313e-16) / std::log(std::abs(z))));
			FilterLines<<<grid, threads, 0, st>>>(c, dims[0], dims[1], dims[2], axis, make_double2(z.real(), z.imag()),
			                                      make_double2(c0.real(), c0.imag()), k0);
			CountLaunch();
		}
		RealTimesGain<<<grid, threads, 0, st>>>(c, static_cast<long long>(count), gain);
		CountLaunch();
		ok = PTB_LAUNCHED();
	}
	if (ok) {
		CentreValues<<<grid, threads, 0, st>>>(c, hdr, dims[0], dims[1], dims[2]);
		CellMonomials<<<grid, threads, 0, st>>>(hdr, coef, dims[0], dims[1], dims[2]);
		CountLaunch(2);
		ok = PTB_LAUNCHED();
	}
	ok = ok && PTB_CUDA(cudaMemcpyAsync(out, coef, cells * 64 * sizeof(double), cudaMemcpyDeviceToHost, st));
	if (c) { cudaFreeAsync(c, st); }
	if (hdr) { cudaFreeAsync(hdr, st); }
	if (coef) { cudaFreeAsync(coef, st); }
	return PTB_CUDA(cudaStreamSynchronize(st)) && ok;
}

}  // namespace ptb
