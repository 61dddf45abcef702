"""Seeded cubic-spline PSF tables in the reference's SplineFit layout (lib/fit/SplineFit.cpp:36-50).

fit_params = [roi, sx, sy, sz, deltaZ, coefficients...] with coefficients SoA [64][sz][sy][sx]: entry
k = i * 16 + j * 4 + m multiplies zf^i * yf^j * xf^m inside a cell (SplineFit.cpp:296-318). The PSF is the
astigmatic Gaussian of the benchmark workloads (optionally with a seeded low-order phase-like distortion), sampled
on a (sz + 3) x (sy + 3) x (sx + 3) grid and turned into per-cell monomial coefficients of the cubic B-spline whose
control points are those samples.
"""
import numpy as np

# cubic B-spline basis in monomial form: B_a(t) = sum_k M[a, k] t^k
_M = np.array([[1, -3, 3, -1], [4, 0, -6, 3], [1, 3, 3, -3], [0, 0, 0, 1]], dtype=np.float64) / 6.0


def psf_samples(sx, sy, sz, dz_nm, sigma0=1.3, distortion=0.0, seed=0):
    """Normalised PSF volume [sz + 3, sy + 3, sx + 3] centred in x / y, z from -sz/2 * dz to +sz/2 * dz."""
    rng = np.random.default_rng(seed)
    zz = (np.arange(sz + 3) - 1 - sz / 2.0) * dz_nm
    yy = np.arange(sy + 3) - 1 - (sy - 1) / 2.0
    xx = np.arange(sx + 3) - 1 - (sx - 1) / 2.0
    u = (zz - 150.0) / 400.0
    v = (zz + 150.0) / 400.0
    gx = sigma0 * np.sqrt(np.maximum(1 + u ** 2 + 0.05 * u ** 3, 1e-3))
    gy = sigma0 * np.sqrt(np.maximum(1 + v ** 2 - 0.05 * v ** 3, 1e-3))
    a, b = rng.normal(0, distortion, 2) if distortion > 0 else (0.0, 0.0)
    vol = np.empty((sz + 3, sy + 3, sx + 3))
    for k in range(sz + 3):
        ex = np.exp(-0.5 * ((xx - a * np.tanh(zz[k] / 400)) / gx[k]) ** 2)
        ey = np.exp(-0.5 * ((yy - b * np.tanh(zz[k] / 400)) / gy[k]) ** 2)
        vol[k] = np.outer(ey, ex) / (2 * np.pi * gx[k] * gy[k])
    return vol


def coefficients(vol):
    """Per-cell monomial coefficients [64, sz, sy, sx] of the B-spline with control points `vol`."""
    sz, sy, sx = (d - 3 for d in vol.shape)
    out = np.zeros((64, sz, sy, sx))
    for i in range(4):
        for j in range(4):
            for m in range(4):
                acc = np.zeros((sz, sy, sx))
                for c in range(4):
                    for b in range(4):
                        for a in range(4):
                            w = _M[c, i] * _M[b, j] * _M[a, m]
                            if w != 0.0:
                                acc += w * vol[c:c + sz, b:b + sy, a:a + sx]
                out[i * 16 + j * 4 + m] = acc
    return out


def fit_params(roi=7, sx=13, sy=13, sz=41, dz_nm=25.0, distortion=0.0, seed=0):
    vol = psf_samples(sx, sy, sz, dz_nm, distortion=distortion, seed=seed)
    coef = coefficients(vol)
    return np.concatenate([[float(roi), float(sx), float(sy), float(sz), dz_nm], coef.ravel()])
