"""The FP64 maximum-likelihood oracle (modes 6-8) against synthetic ground truth.

The GPU fits of modes 6-8 are checked against this oracle; here the oracle itself is checked against the emitters
that rendered the data. Isolated emitters (one per 24 x 24 pixel cell) are drawn from each mode's own model with the
benchmark camera (ADU = 100 + 2 x Poisson(photons)) and fitted one by one. For every parameter the normalised error
(estimate - truth) / CRLB must have |mean| <= 0.1 and a standard deviation within 15 % of 1 over >= 2000 fits: an
unbiased, efficient estimator whose reported CRLB matches its spread. A modelling error shared by the oracle and the
GPU (pixel integration, photon conversion, width model, spline indexing) would show up here as bias or as a spread
the CRLB does not explain.
"""
import math

import numpy as np
import pytest
from scipy.special import erf

ASTIG = [150.0, 400.0, 0.05, 0.0, 1.3 * 160, -150.0, 400.0, -0.05, 0.0, 1.3 * 160]
CELL = 24
GRID = 24  # emitters per row and column of one frame: 576 per frame


def _erf_profile(centers, x, s):
    """Fraction of a unit 1D Gaussian (mean x, sd s) falling in the pixels [c - 0.5, c + 0.5]."""
    return 0.5 * (erf((centers + 0.5 - x) / (math.sqrt(2) * s)) - erf((centers - 0.5 - x) / (math.sqrt(2) * s)))


def _astig_sigma(m, z):
    u = (z - m[0]) / m[1]
    return m[4] / 160.0 * np.sqrt(1 + u * u + m[2] * u ** 3 + m[3] * u ** 4)


def _spline_psf(coef, sx, sy, sz, X, Y, Z):
    """The spline model of mode 8 at table coordinates (cells are clamped like the fit's)."""
    ix = np.clip(np.floor(X).astype(int), 0, sx - 1)
    iy = np.clip(np.floor(Y).astype(int), 0, sy - 1)
    iz = np.clip(np.floor(Z).astype(int), 0, sz - 1)
    fx, fy, fz = X - ix, Y - iy, Z - iz
    c = coef.reshape(64, sz, sy, sx)[:, iz, iy, ix]
    v = np.zeros_like(X)
    for i in range(4):
        for j in range(4):
            for m in range(4):
                v += c[i * 16 + j * 4 + m] * fz ** i * fy ** j * fx ** m
    return v


def _frames(model, n_frames, rng, spline=None):
    """Frames of isolated emitters and their truth: columns x, y, photons, bg, shape (sigma px | z nm | z cells)."""
    size = CELL * GRID
    frames, truth = [], []
    for _ in range(n_frames):
        bg = rng.uniform(10.0, 40.0)
        mu = np.full((size, size), bg)
        for gy in range(GRID):
            for gx in range(GRID):
                x = gx * CELL + CELL / 2 + rng.uniform(-0.5, 0.5)
                y = gy * CELL + CELL / 2 + rng.uniform(-0.5, 0.5)
                ph = math.exp(rng.uniform(math.log(1000), math.log(5000)))
                xs = np.arange(int(x) - 8, int(x) + 9)
                ys = np.arange(int(y) - 8, int(y) + 9)
                if model == 6:
                    s = rng.uniform(1.0, 1.6)
                    patch = np.outer(_erf_profile(ys, y, s), _erf_profile(xs, x, s))
                    shape = s
                elif model == 7:
                    z = rng.uniform(-400.0, 400.0)
                    patch = np.outer(_erf_profile(ys, y, _astig_sigma(ASTIG[5:], z)), _erf_profile(xs, x, _astig_sigma(ASTIG[:5], z)))
                    shape = z
                else:
                    coef, sx, sy, sz = spline
                    z = sz / 2.0 + rng.uniform(-15.0, 15.0)
                    X = (sx - 1) / 2.0 + xs[None, :] - x
                    Y = (sy - 1) / 2.0 + ys[:, None] - y
                    X, Y = np.broadcast_arrays(X, Y)
                    patch = _spline_psf(coef, sx, sy, sz, X, Y, np.full(X.shape, z))
                    shape = z
                mu[np.ix_(ys, xs)] += ph * patch
                truth.append((x, y, ph, bg, shape))
        frames.append(np.clip(100 + 2 * rng.poisson(mu), 0, 65535).astype(np.uint16))
    return frames, np.array(truth)


def _params(model, spline=None):
    if model == 6:
        return np.array([7.0, 1.3, 100.0, 2.0, 30.0, 0.0])
    if model == 7:
        return np.array([11.0, 160.0] + ASTIG + [100.0, 2.0, 30.0, -600.0, 600.0, 0.0])
    coef, sx, sy, sz = spline
    return np.concatenate([[13.0, sx, sy, sz, 20.0, 100.0, 2.0, 30.0, 0.0], coef])


@pytest.mark.parametrize("model", [6, 7, 8])
def test_oracle_mle_recovers_ground_truth(orc, model):
    rng = np.random.default_rng(600 + model)
    spline = None
    if model == 8:
        import spline_table
        sx = sy = 25
        sz = 61
        p = spline_table.fit_params(roi=13, sx=sx, sy=sy, sz=sz, dz_nm=20.0, distortion=0.2, seed=9)
        spline = (p[5:], sx, sy, sz)
    frames, truth = _frames(model, 4, rng, spline)
    params = _params(model, spline)
    est, crlb = [], []
    k = 0
    for fr in frames:
        for _ in range(GRID * GRID):
            x, y = truth[k, 0], truth[k, 1]
            # the candidate: the emitter's pixel, as a segmentation centroid would give it
            cx, cy = math.floor(x) + 0.5, math.floor(y) + 0.5
            st, t, c, _ = orc.mle_fit_one(fr, cx, cy, model, params)
            assert st == 1
            ux, uy = math.floor(cx), math.floor(cy)
            est.append([t[2] + ux, t[3] + uy, t[1], t[0], t[4]])
            crlb.append([c[2], c[3], c[1], c[0], c[4]])
            k += 1
    est, crlb = np.array(est), np.array(crlb)
    assert est.shape[0] >= 2000
    zscore = (est - truth) / crlb
    names = ["x", "y", "photons", "background", {6: "sigma", 7: "z", 8: "z"}[model]]
    report = {n: (float(zscore[:, i].mean()), float(zscore[:, i].std())) for i, n in enumerate(names)}
    print("model", model, "fits", est.shape[0], "(mean, sd) of (estimate - truth) / CRLB:", report)
    for n, (m, s) in report.items():
        assert abs(m) <= 0.1 and 0.85 <= s <= 1.15, (model, n, m, s)
