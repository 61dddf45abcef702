"""PTB_LocalizationTiff: a TIFF stack localized from the file (frames read into pinned staging while the previous
chunk computes) gives the same rows, bit for bit, as Localization over the same frames in memory; with one chunk
and with many (a small device budget, so the two staging slots are refilled from the file many times).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import tiffgen
from conftest import GAUSS_PARAMS

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MLE6 = np.array([7.0, 1.3, 100.0, 2.0, 20, 0.0])

CHILD = r"""
import os, sys
import numpy as np
sys.path[:0] = [os.path.join(sys.argv[1], "palmtracer-cpp_b200"), os.path.join(sys.argv[1], "tests")]
import ptb
data = np.load(sys.argv[2])
out = {}
for key in ("g", "m"):
    out[key] = ptb.localization_tiff(sys.argv[4], float(data["thr"]), 0.0, int(data["fit_" + key]), data["params_" + key])
np.savez(sys.argv[3], **out)
"""


def test_tiff_stack_equals_in_memory_stack(lib, orc, tmp_path, monkeypatch):
    import synth
    monkeypatch.setenv("PTB_MLE_LANES", "1")
    s, _ = synth.stack("c1", frames=9, seed=404)
    thr = synth.mad_threshold(orc.planes(s[0])[1])
    path = str(tmp_path / "stack.tif")
    tiffgen.write(path, list(s), big_endian=True, rows_per_strip=3)
    assert lib.tiff_info(path) == (s.shape[2], s.shape[1], s.shape[0])
    ref = {"g": lib.localization(s, thr, 0.0, 2, GAUSS_PARAMS), "m": lib.localization(s, thr, 0.0, 6, MLE6)}
    for key, fit, params in (("g", 2, GAUSS_PARAMS), ("m", 6, MLE6)):
        got = lib.localization_tiff(path, thr, 0.0, fit, params)
        assert ref[key].shape[0] > 100 and got.shape == ref[key].shape and np.array_equal(got, ref[key]), key
    # many chunks: the file is read chunk by chunk into the two pinned staging slots
    inp, outp = tmp_path / "in.npz", tmp_path / "out.npz"
    np.savez(inp, thr=thr, fit_g=2, params_g=GAUSS_PARAMS, fit_m=6, params_m=MLE6)
    env = dict(os.environ, PTB_WORKSPACE_MB="8", PTB_MLE_LANES="1")
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, str(inp), str(outp), path], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    got = np.load(outp)
    for key in ("g", "m"):
        assert got[key].shape == ref[key].shape and np.array_equal(got[key], ref[key]), key


def test_tiff_errors_reach_the_caller(lib, tmp_path):
    path = str(tmp_path / "bad.tif")
    tiffgen.write(path, [np.zeros((16, 16), np.uint8)], bits=8)
    out = np.zeros(18 * 100)
    n = lib.load().PTB_LocalizationTiff(os.fsencode(path), out.ctypes.data_as(lib._f64p), out.size, 100.0, 0.0, 2,
                                        GAUSS_PARAMS.ctypes.data_as(lib._f64p))
    assert n == 0 and "16 bits" in lib.last_error()
