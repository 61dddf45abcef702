"""ctypes access to the CPU oracle libraries (test infrastructure only).

Two libraries share one calling convention:
  * oracle/liboracle.so      - the C++ restatement in oracle/pt_oracle.cpp (prefix ``orc_``)
  * oracle/_ref/libptref.so  - the unmodified reference sources + oracle/ref_shim.cpp (prefix ``ref_``)

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this module, as the checker.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libptref.so")
COLS = 18

_u16p = ctypes.POINTER(ctypes.c_uint16)
_f64p = ctypes.POINTER(ctypes.c_double)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64 = ctypes.c_uint64
_f64 = ctypes.c_double


def _ptr(a, t):
    return a.ctypes.data_as(t)


class CpuLib:
    """One of the two CPU libraries; ``prefix`` selects the symbol family."""

    def __init__(self, path, prefix):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.path = path
        self.lib = ctypes.CDLL(path)
        self.prefix = prefix
        L = self.lib
        self._loc = getattr(L, prefix + "Localization")
        self._loc.restype = _u64
        self._loc.argtypes = [_u16p, _f64p, _u64, _u64, _u64, _u64, _f64, _f64, _u64, _f64p]
        self._fit = getattr(L, prefix + "Fitting")
        self._fit.restype = _u64
        self._fit.argtypes = [_u16p, _f64p, _u64, _f64p, _u64, _u64, _u64, _u64, _u64, _f64p]
        self._wav = getattr(L, prefix + "Wavelett")
        self._wav.restype = None
        self._wav.argtypes = [_u16p, _f64p, _u64, _u64, _u64, _u64]
        self._thr = getattr(L, prefix + "AutoThreshold")
        self._thr.restype = _f64
        self._thr.argtypes = [_u16p, _u64, _u64, _f64p]
        self._planes = getattr(L, prefix + "Planes")
        self._planes.restype = None
        self._planes.argtypes = [_u16p, _u64, _u64, _f64p]
        self._cand = getattr(L, prefix + "Candidates")
        self._cand.restype = _u64
        self._cand.argtypes = [_u16p, _u64, _u64, _f64, _f64, _f64p, _u64]
        self._candp = getattr(L, prefix + "CandidatesFromPotential")
        self._candp.restype = _u64
        self._candp.argtypes = [_f64p, _u64, _u64, _f64, _f64, _f64p, _u64]
        self._threads = getattr(L, prefix + "SetThreads")
        self._threads.restype = None
        self._threads.argtypes = [ctypes.c_int]

    def astig_estimation(self, sigmas, pixel_size, model, zmax):
        """Astigmatism3DEstimation: [n, 2] (sigma_x, sigma_y) px -> [n, 2] (z nm, score)."""
        f = getattr(self.lib, self.prefix + "Astig3DEstimation")
        f.restype = None
        f.argtypes = [_f64p, _f64p, _u64, _f64, _f64p, _f64]
        sigmas = np.ascontiguousarray(sigmas, dtype=np.float64).reshape(-1, 2)
        out = np.zeros_like(sigmas)
        model = np.ascontiguousarray(model, dtype=np.float64)
        f(_ptr(sigmas, _f64p), _ptr(out, _f64p), sigmas.shape[0], pixel_size, _ptr(model, _f64p), zmax)
        return out

    def tracking(self, points, max_distance):
        """Tracking: points [n, 4] (Id, Plane, X, Y) -> [n, 2] uint64 (Id, Track) in (Plane, Id) order."""
        f = getattr(self.lib, self.prefix + "Tracking")
        f.restype = _u64
        f.argtypes = [_f64p, ctypes.POINTER(ctypes.c_uint64), _u64, _f64]
        points = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 4)
        out = np.zeros((points.shape[0], 2), dtype=np.uint64)
        if points.shape[0]:
            f(_ptr(points, _f64p), out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), points.shape[0], max_distance)
        return out

    def set_threads(self, n):
        self._threads(int(n))

    def localization(self, stack, thr, ratio, fit, params, capacity_doubles=None):
        stack = np.ascontiguousarray(stack, dtype=np.uint16)
        if stack.ndim == 2:
            stack = stack[None]
        z, h, w = stack.shape
        if capacity_doubles is None:
            capacity_doubles = ((h * w) // 5 + 1) * z * COLS
        out = np.full(max(capacity_doubles, 1), -12345.0)
        params = np.ascontiguousarray(params, dtype=np.float64)
        n = self._loc(_ptr(stack, _u16p), _ptr(out, _f64p), capacity_doubles, h, w, z, thr, ratio, fit, _ptr(params, _f64p))
        return out[:n].reshape(-1, COLS).copy()

    def fitting(self, stack, positions, fit, params):
        stack = np.ascontiguousarray(stack, dtype=np.uint16)
        if stack.ndim == 2:
            stack = stack[None]
        z, h, w = stack.shape
        positions = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 6)
        n = positions.shape[0]
        out = np.zeros(max(n, 1) * COLS)
        params = np.ascontiguousarray(params, dtype=np.float64)
        k = self._fit(_ptr(stack, _u16p), _ptr(positions, _f64p), n, _ptr(out, _f64p), out.size, h, w, z, fit, _ptr(params, _f64p))
        return out[:k].reshape(-1, COLS).copy()

    def wavelett(self, stack, level):
        stack = np.ascontiguousarray(stack, dtype=np.uint16)
        if stack.ndim == 2:
            stack = stack[None]
        z, h, w = stack.shape
        out = np.zeros((z, h, w))
        self._wav(_ptr(stack, _u16p), _ptr(out, _f64p), h, w, z, level)
        return out

    def auto_threshold(self, frame, params):
        frame = np.ascontiguousarray(frame, dtype=np.uint16)
        h, w = frame.shape[-2:]
        params = np.ascontiguousarray(params, dtype=np.float64)
        return self._thr(_ptr(frame, _u16p), h, w, _ptr(params, _f64p))

    def planes(self, frame):
        frame = np.ascontiguousarray(frame, dtype=np.uint16)
        h, w = frame.shape
        out = np.zeros((3, h, w))
        self._planes(_ptr(frame, _u16p), h, w, _ptr(out, _f64p))
        return out

    def candidates(self, frame, thr, ratio):
        frame = np.ascontiguousarray(frame, dtype=np.uint16)
        h, w = frame.shape
        cap = h * w // 4 + 16
        rows = np.zeros((cap, 4))
        n = self._cand(_ptr(frame, _u16p), h, w, thr, ratio, _ptr(rows, _f64p), cap)
        return rows[:min(n, cap)].copy()

    def candidates_from_potential(self, potential, thr, ratio):
        potential = np.ascontiguousarray(potential, dtype=np.float64)
        h, w = potential.shape
        cap = h * w // 4 + 16
        rows = np.zeros((cap, 4))
        n = self._candp(_ptr(potential, _f64p), h, w, thr, ratio, _ptr(rows, _f64p), cap)
        return rows[:min(n, cap)].copy()


class OracleLib(CpuLib):
    def __init__(self, path=ORACLE_SO):
        super().__init__(path, "orc_")
        self._labels = self.lib.orc_Labels
        self._labels.restype = _u64
        self._labels.argtypes = [_u16p, _u64, _u64, _f64, _f64, _u32p]

    def labels(self, frame, thr, ratio):
        frame = np.ascontiguousarray(frame, dtype=np.uint16)
        h, w = frame.shape
        out = np.zeros((h, w), dtype=np.uint32)
        self._labels(_ptr(frame, _u16p), h, w, thr, ratio, _ptr(out, _u32p))
        return out

    def mle_evaluate(self, frame, cx, cy, fit, params, theta):
        """FP64 deviance, gradient and exact Hessian of the maximum-likelihood objective at theta (local to the ROI
        centre floor(cx), floor(cy)); None when the ROI crosses the border."""
        frame = np.ascontiguousarray(frame, dtype=np.uint16)
        params = np.ascontiguousarray(params, dtype=np.float64)
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        d, g, h = np.zeros(1), np.zeros(5), np.zeros(25)
        f = self.lib.orc_MleEvaluate
        f.restype = ctypes.c_int
        f.argtypes = [_u16p, _u64, _u64, _f64, _f64, _u64, _f64p, _f64p, _f64p, _f64p, _f64p]
        if not f(_ptr(frame, _u16p), frame.shape[0], frame.shape[1], cx, cy, fit, _ptr(params, _f64p), _ptr(theta, _f64p),
                 _ptr(d, _f64p), _ptr(g, _f64p), _ptr(h, _f64p)):
            return None
        return float(d[0]), g, h.reshape(5, 5)

    def spline_coefficients(self, volume, lam=None, with_centres=False):
        """The spline calibration's coefficient table of a PSF volume [nz, ny, nx]: [cells, 64] in the reference's
        layout (cells z, y, x); with_centres also returns the spline's values at the voxel centres."""
        volume = np.ascontiguousarray(volume, dtype=np.float64)
        nz, ny, nx = volume.shape
        out = np.zeros(((nz - 1) * (ny - 1) * (nx - 1), 64))
        hdr = np.zeros_like(volume)
        f = self.lib.orc_SplineCoefficients
        f.restype = _u64
        f.argtypes = [_f64p, _u64, _u64, _u64, _f64p, _f64p, _f64p]
        lam_p = None
        if lam is not None:
            lam = np.ascontiguousarray(lam, dtype=np.float64)
            lam_p = _ptr(lam, _f64p)
        n = f(_ptr(volume, _f64p), nx, ny, nz, lam_p, _ptr(out, _f64p), _ptr(hdr, _f64p))
        if n == 0 or n != out.size:
            raise RuntimeError("orc_SplineCoefficients failed")
        return (out, hdr) if with_centres else out

    def mle_fit_one(self, frame, cx, cy, fit, params):
        """(status, theta, crlb, deviance) of one candidate's fit: status 1 success, 2 failed, 0 border."""
        frame = np.ascontiguousarray(frame, dtype=np.uint16)
        params = np.ascontiguousarray(params, dtype=np.float64)
        t, c, d = np.zeros(5), np.zeros(5), np.zeros(1)
        f = self.lib.orc_MleFitOne
        f.restype = ctypes.c_int
        f.argtypes = [_u16p, _u64, _u64, _f64, _f64, _u64, _f64p, _f64p, _f64p, _f64p]
        st = f(_ptr(frame, _u16p), frame.shape[0], frame.shape[1], cx, cy, fit, _ptr(params, _f64p), _ptr(t, _f64p),
               _ptr(c, _f64p), _ptr(d, _f64p))
        return st, t, c, float(d[0])


class RefLib(CpuLib):
    def __init__(self, path=REF_SO):
        super().__init__(path, "ref_")


def oracle():
    return OracleLib()


def reference():
    """The reference built from source, or None when oracle/_ref has not been built."""
    return RefLib() if os.path.exists(REF_SO) else None


def reference_root():
    """The reference source tree (for tests that read its fixtures): $PTB_REFERENCE_ROOT, else the tree oracle/_ref was
    built from; None when neither exists on this machine."""
    root = os.environ.get("PTB_REFERENCE_ROOT")
    if not root:
        rec = os.path.join(HERE, "_ref", "reference_root.txt")
        if os.path.exists(rec):
            with open(rec) as f:
                root = f.read().strip()
    return root if root and os.path.isdir(root) else None
