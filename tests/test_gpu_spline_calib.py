"""PTB_SplineCoefficients (the spline calibration's coefficient step on the GPU) against the oracle restatement of
lib/signal_processing/BSpline3D.cpp, and its table driving the spline fits.

The GPU writes the table in the fits' layout (SoA [64][cell]); the oracle in the reference's ([cell][64]). The two
compute the same polynomials by different FP64 routes (the reference's 64 x 64 solve against a direct basis change),
so they agree to rounding: 1e-9 of the largest coefficient.
"""
import os

import numpy as np
import pytest

from compare import match_rows
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _bead():
    b = np.load(os.path.join(GOLDEN, "beads.npz"))["bead"].astype(np.float64)
    b -= np.median(b)
    return b / b.max()


def _psf():
    import spline_table
    return spline_table.psf_samples(12, 10, 14, 50.0, distortion=0.2, seed=3)


@pytest.mark.parametrize("which,lam", [("psf", None), ("bead", None), ("bead", [0.0, 0.0, 10.0]), ("psf", [0.5, 0.25, 2.0])])
def test_table_matches_oracle(lib, orc, which, lam):
    vol = _psf() if which == "psf" else _bead()
    gpu = lib.spline_coefficients(vol, lam)
    cpu = orc.spline_coefficients(vol, lam)
    assert gpu.shape == (64,) + tuple(d - 1 for d in vol.shape)
    soa = np.ascontiguousarray(cpu.T).reshape(gpu.shape)
    scale = np.max(np.abs(cpu))
    assert np.max(np.abs(gpu - soa)) <= 1e-9 * scale, float(np.max(np.abs(gpu - soa)) / scale)


def test_table_drives_the_spline_fits(lib, orc, stacks):
    """The produced table is a ready fit_params table: mode-5 fits with it agree with the oracle's."""
    table = lib.spline_coefficients(_psf())
    sz, sy, sx = table.shape[1:]
    params = np.concatenate([[7.0, sx, sy, sz, 50.0], table.ravel()])
    st = stacks["stack"][:2]
    a = lib.localization(st, 103.6, 0.0, 5, params)
    b = orc.localization(st, 103.6, 0.0, 5, params)
    assert a.shape == b.shape and a.shape[0] > 0
    assert match_rows(a, b, atol=1e-6, rtol=1e-6)[0] == 0


def test_degenerate_volume_is_rejected(lib):
    with pytest.raises(RuntimeError):
        lib.spline_coefficients(np.zeros((1, 4, 4)))
