"""Spline calibration's coefficient step (the oracle restatement of lib/signal_processing/BSpline3D.cpp; no GPU).

The reference's B-spline code cannot be built here (lib/signal_processing/Interpolation.cpp includes FFTW, which
this image lacks) and its tests hold no known answers for the table (Tests_CPU/test_sp_BSpline.cpp,
test_sp_Spline.cpp:395-450), so the restatement is checked through the properties the algorithm guarantees: the
unregularised prefilter makes the spline interpolate the volume, a regularised axis is smoothed, the poles solve their
polynomial, and the per-cell polynomials join with continuous values and first and second derivatives (a cubic
spline). Inputs: a synthetic astigmatic PSF and a crop of the reference's own bead stack (Tests_CPU/Input/Beads.tiff).
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN


def _bead():
    b = np.load(os.path.join(GOLDEN, "beads.npz"))["bead"].astype(np.float64)
    b -= np.median(b)
    return b / b.max()


def _psf():
    import spline_table
    return spline_table.psf_samples(12, 10, 14, 50.0, distortion=0.2, seed=3)


def _poly(coef_cell, zf, yf, xf):
    """Value and first / second derivatives along each axis of one cell's polynomial at (zf, yf, xf)."""
    c = coef_cell.reshape(4, 4, 4)  # [z power][y power][x power]
    pw = lambda t, d: np.array([0 if p < d else np.prod(range(p - d + 1, p + 1)) * t ** (p - d) for p in range(4)], float)
    out = {}
    for name, (dz, dy, dx) in {"v": (0, 0, 0), "dz": (1, 0, 0), "dy": (0, 1, 0), "dx": (0, 0, 1),
                               "zz": (2, 0, 0), "yy": (0, 2, 0), "xx": (0, 0, 2)}.items():
        out[name] = float(np.einsum("lmn,l,m,n->", c, pw(zf, dz), pw(yf, dy), pw(xf, dx)))
    return out


@pytest.mark.parametrize("which", ["psf", "bead"])
def test_unregularised_spline_interpolates_the_volume(orc, which):
    vol = _psf() if which == "psf" else _bead()
    _, hdr = orc.spline_coefficients(vol, with_centres=True)
    assert np.max(np.abs(hdr - vol)) <= 1e-10 * np.max(np.abs(vol))


def test_regularised_axis_is_smoothed(orc):
    vol = _bead()
    _, hdr0 = orc.spline_coefficients(vol, with_centres=True)
    _, hdr1 = orc.spline_coefficients(vol, lam=[0.0, 0.0, 100.0 / 10.0], with_centres=True)  # calibration: 100 / dz
    rough = lambda v, ax: float(np.sum(np.diff(v, 2, axis=ax) ** 2))
    assert rough(hdr1, 0) < 0.5 * rough(hdr0, 0)        # z (axis 0 of [z, y, x]) smoothed
    assert abs(rough(hdr1, 2) / rough(hdr0, 2) - 1) < 0.5  # x barely changed


def test_regularised_poles_solve_their_polynomial():
    """The closed form the GPU uses (w = z + 1/z) and the quartic: both poles inside the unit circle, roots of it."""
    for lam in (0.01, 0.1, 1.0, 10.0, 100.0):
        b, c = -4 + 1 / (6 * lam), 6 + 2 / (3 * lam)
        roots = np.roots([1, b, c, b, 1])
        inside = roots[np.abs(roots) <= 1]
        assert len(inside) == 2
        for z in inside:
            assert abs(np.polyval([1, b, c, b, 1], z)) < 1e-10


@pytest.mark.parametrize("lam", [None, [0.0, 0.0, 10.0]])
def test_cells_join_as_a_cubic_spline(orc, lam):
    vol = _bead()[:20, :12, :12]
    coef = orc.spline_coefficients(vol, lam=lam)
    nz, ny, nx = (d - 1 for d in vol.shape)
    cell = lambda z, y, x: coef[(z * ny + y) * nx + x]
    scale = np.max(np.abs(coef))
    rng = np.random.default_rng(1)
    for _ in range(40):
        z, y, x = rng.integers(0, nz - 1), rng.integers(0, ny - 1), rng.integers(0, nx - 1)
        a, b = rng.uniform(0, 1, 2)
        for axis in range(3):
            if axis == 0:
                left, right = _poly(cell(z, y, x), 1.0, a, b), _poly(cell(z + 1, y, x), 0.0, a, b)
            elif axis == 1:
                left, right = _poly(cell(z, y, x), a, 1.0, b), _poly(cell(z, y + 1, x), a, 0.0, b)
            else:
                left, right = _poly(cell(z, y, x), a, b, 1.0), _poly(cell(z, y, x + 1), a, b, 0.0)
            for k in ("v", "dz", "dy", "dx", "zz", "yy", "xx"):
                assert abs(left[k] - right[k]) <= 1e-9 * scale * 10, (axis, k, left[k], right[k])


def test_degenerate_dimensions_are_rejected(orc):
    with pytest.raises(RuntimeError):
        orc.spline_coefficients(np.zeros((1, 5, 5)))
