"""ctypes binding of libpalmtracer_b200.so for Python callers (tests, benchmark, the reference front-end).

The functions mirror the C ABI in include/palmtracer_b200.h one for one; numpy arrays are passed as host buffers.
Loading fails loudly when the library has not been built: there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpalmtracer_b200.so")
COLS = 18

# every symbol the public header declares
EXPORTS = ["Localization", "Fitting", "Wavelett", "AutoThreshold", "Astigmatism3DEstimation", "PTB_LocalizationDevice",
           "PTB_SetSegmentationMode", "PTB_SetFitPrecision", "PTB_LastError", "PTB_KernelLaunchCount",
           "PTB_SetProfiling", "PTB_StageTimes", "PTB_MleEvaluations", "PTB_GraphStats", "PTB_SegmentationStats", "PTB_EnginePoolStats",
           "PTB_MleMappings", "PTB_DetectStagingStats",
           "PTB_MeasureFmaPeak", "PTB_FittingDeviceNoAlloc",
           "PTB_ServerStart", "PTB_SubmitStack", "PTB_PollStack", "PTB_StackResult", "PTB_ServerStop", "PTB_ServerFuseStats",
           "PTB_TiffInfo", "PTB_TiffRead", "PTB_LocalizationTiff", "Tracking", "PTB_TrackingDevice", "PTB_SplineCoefficients"]

_u16p = ctypes.POINTER(ctypes.c_uint16)
_f64p = ctypes.POINTER(ctypes.c_double)
_u64 = ctypes.c_uint64
_f64 = ctypes.c_double

_lib = None


def load(path=LIB_PATH):
    """Loads the library once (raises OSError when it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError("libpalmtracer_b200.so not built: run python palmtracer-cpp_b200/build.py (%s)" % path)
    L = ctypes.CDLL(path)
    L.Localization.restype = _u64
    L.Localization.argtypes = [_u16p, _f64p, _u64, _u64, _u64, _u64, _f64, _f64, _u64, _f64p]
    L.Fitting.restype = _u64
    L.Fitting.argtypes = [_u16p, _f64p, _u64, _f64p, _u64, _u64, _u64, _u64, _u64, _f64p]
    L.Wavelett.restype = None
    L.Wavelett.argtypes = [_u16p, _f64p, _u64, _u64, _u64, _u64]
    L.AutoThreshold.restype = _f64
    L.AutoThreshold.argtypes = [_u16p, _u64, _u64, _f64p]
    L.Astigmatism3DEstimation.restype = None
    L.Astigmatism3DEstimation.argtypes = [_f64p, _f64p, _u64, _f64, _f64p, _f64]
    L.PTB_LocalizationDevice.restype = _u64
    L.PTB_LocalizationDevice.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _u64, _u64, _u64, _u64, _f64, _f64, _u64, _f64p,
                                         ctypes.c_void_p]
    L.PTB_SetSegmentationMode.restype = ctypes.c_int
    L.PTB_SetSegmentationMode.argtypes = [ctypes.c_int]
    L.PTB_SetFitPrecision.restype = ctypes.c_int
    L.PTB_SetFitPrecision.argtypes = [ctypes.c_int]
    L.PTB_LastError.restype = ctypes.c_char_p
    L.PTB_LastError.argtypes = []
    L.PTB_KernelLaunchCount.restype = _u64
    L.PTB_KernelLaunchCount.argtypes = []
    L.PTB_SetProfiling.restype = ctypes.c_int
    L.PTB_SetProfiling.argtypes = [ctypes.c_int]
    L.PTB_StageTimes.restype = None
    L.PTB_StageTimes.argtypes = [_f64p, ctypes.POINTER(ctypes.c_uint64), ctypes.c_int]
    L.PTB_MleEvaluations.restype = None
    L.PTB_MleEvaluations.argtypes = [ctypes.POINTER(ctypes.c_uint64), ctypes.c_int]
    L.Tracking.restype = None
    L.Tracking.argtypes = [_f64p, ctypes.POINTER(_u64), _u64, _f64]
    L.PTB_TrackingDevice.restype = _u64
    L.PTB_TrackingDevice.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _u64, _f64, ctypes.c_void_p]
    L.PTB_TiffInfo.restype = ctypes.c_int
    L.PTB_TiffInfo.argtypes = [ctypes.c_char_p, ctypes.POINTER(_u64), ctypes.POINTER(_u64), ctypes.POINTER(_u64)]
    L.PTB_TiffRead.restype = _u64
    L.PTB_TiffRead.argtypes = [ctypes.c_char_p, _u16p, _u64, _u64]
    L.PTB_LocalizationTiff.restype = _u64
    L.PTB_LocalizationTiff.argtypes = [ctypes.c_char_p, _f64p, _u64, _f64, _f64, _u64, _f64p]
    L.PTB_DetectStagingStats.restype = None
    L.PTB_DetectStagingStats.argtypes = [ctypes.POINTER(ctypes.c_uint64), ctypes.c_int]
    L.PTB_GraphStats.restype = None
    L.PTB_GraphStats.argtypes = [ctypes.POINTER(ctypes.c_uint64), ctypes.c_int]
    L.PTB_SegmentationStats.restype = None
    L.PTB_SegmentationStats.argtypes = [ctypes.POINTER(ctypes.c_uint64), ctypes.c_int]
    L.PTB_EnginePoolStats.restype = None
    L.PTB_EnginePoolStats.argtypes = [ctypes.POINTER(ctypes.c_uint64), ctypes.c_int]
    L.PTB_MleMappings.restype = ctypes.c_int
    L.PTB_MleMappings.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_int]
    L.PTB_SplineCoefficients.restype = _u64
    L.PTB_SplineCoefficients.argtypes = [_f64p, _u64, _u64, _u64, _f64p, _f64p]
    L.PTB_ServerFuseStats.restype = None
    L.PTB_ServerFuseStats.argtypes = [ctypes.POINTER(ctypes.c_uint64), ctypes.c_int]
    L.PTB_FittingDeviceNoAlloc.restype = _u64
    L.PTB_FittingDeviceNoAlloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _u64, ctypes.c_void_p, _u64, _u64, _u64, _u64,
                                           _f64p, ctypes.c_void_p]
    L.PTB_ServerStart.restype = ctypes.c_int
    L.PTB_ServerStart.argtypes = [ctypes.c_int, _u64]
    L.PTB_SubmitStack.restype = _u64
    L.PTB_SubmitStack.argtypes = [_u16p, _f64p, _u64, _u64, _u64, _u64, _f64, _f64, _u64, _f64p]
    L.PTB_PollStack.restype = ctypes.c_int
    L.PTB_PollStack.argtypes = [_u64]
    L.PTB_StackResult.restype = ctypes.c_int64
    L.PTB_StackResult.argtypes = [_u64, _f64p]
    L.PTB_ServerStop.restype = None
    L.PTB_ServerStop.argtypes = []
    L.PTB_MeasureFmaPeak.restype = _f64
    L.PTB_MeasureFmaPeak.argtypes = [ctypes.c_int]
    _lib = L
    return L


def _stack(stack):
    stack = np.ascontiguousarray(stack, dtype=np.uint16)
    if stack.ndim == 2:
        stack = stack[None]
    return stack


def last_error():
    return load().PTB_LastError().decode()


def localization(stack, thr, ratio, fit, params, capacity_doubles=None):
    """Localization over a host stack; returns the [n, 18] float64 rows."""
    L = load()
    stack = _stack(stack)
    z, h, w = stack.shape
    if capacity_doubles is None:
        capacity_doubles = ((h * w) // 5 + 1) * z * COLS
    out = np.full(max(capacity_doubles, 1), -12345.0)
    params = np.ascontiguousarray(params, dtype=np.float64)
    n = L.Localization(stack.ctypes.data_as(_u16p), out.ctypes.data_as(_f64p), capacity_doubles, h, w, z, thr, ratio, fit,
                       params.ctypes.data_as(_f64p))
    return out[:n].reshape(-1, COLS).copy()


def localization_raw(stack, out, thr, ratio, fit, params):
    """Localization into a caller-given float64 buffer (its size is the capacity); returns doubles written."""
    L = load()
    z, h, w = stack.shape
    params = np.ascontiguousarray(params, dtype=np.float64)
    return L.Localization(stack.ctypes.data_as(_u16p), out.ctypes.data_as(_f64p), out.size, h, w, z, thr, ratio, fit,
                          params.ctypes.data_as(_f64p))


def fitting(stack, positions, fit, params):
    L = load()
    stack = _stack(stack)
    z, h, w = stack.shape
    positions = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 6)
    n = positions.shape[0]
    out = np.zeros(max(n, 1) * COLS)
    params = np.ascontiguousarray(params, dtype=np.float64)
    k = L.Fitting(stack.ctypes.data_as(_u16p), positions.ctypes.data_as(_f64p), n, out.ctypes.data_as(_f64p), out.size, h, w, z,
                  fit, params.ctypes.data_as(_f64p))
    return out[:k].reshape(-1, COLS).copy()


def wavelett(stack, level):
    L = load()
    stack = _stack(stack)
    z, h, w = stack.shape
    out = np.zeros((z, h, w))
    L.Wavelett(stack.ctypes.data_as(_u16p), out.ctypes.data_as(_f64p), h, w, z, level)
    return out


def auto_threshold(frame, params):
    L = load()
    frame = np.ascontiguousarray(frame, dtype=np.uint16)
    h, w = frame.shape[-2:]
    params = np.ascontiguousarray(params, dtype=np.float64)
    return L.AutoThreshold(frame.ctypes.data_as(_u16p), h, w, params.ctypes.data_as(_f64p))


def astig_estimation(sigmas, pixel_size, model, zmax):
    """Astigmatism3DEstimation: [n, 2] (sigma_x, sigma_y) px -> [n, 2] (z nm, score)."""
    sigmas = np.ascontiguousarray(sigmas, dtype=np.float64).reshape(-1, 2)
    out = np.zeros_like(sigmas)
    model = np.ascontiguousarray(model, dtype=np.float64)
    load().Astigmatism3DEstimation(sigmas.ctypes.data_as(_f64p), out.ctypes.data_as(_f64p), sigmas.shape[0], pixel_size,
                                   model.ctypes.data_as(_f64p), zmax)
    return out


def localization_device(d_input_ptr, d_output_ptr, capacity_doubles, shape, thr, ratio, fit, params, stream_ptr=0):
    """Device-buffer variant: pointers are CUDA device addresses (e.g. torch tensor.data_ptr())."""
    L = load()
    z, h, w = shape
    params = np.ascontiguousarray(params, dtype=np.float64)
    return L.PTB_LocalizationDevice(ctypes.c_void_p(d_input_ptr), ctypes.c_void_p(d_output_ptr), capacity_doubles, h, w, z,
                                    thr, ratio, fit, params.ctypes.data_as(_f64p), ctypes.c_void_p(stream_ptr))


def set_segmentation_mode(mode):
    return load().PTB_SetSegmentationMode(int(mode))


def set_fit_precision(mode):
    return load().PTB_SetFitPrecision(int(mode))


def launch_count():
    return load().PTB_KernelLaunchCount()


STAGES = ["detect", "segment", "fit", "finish", "copies", "fit_init", "fit_lm", "fit_polish", "fit_final"]


def set_profiling(enable):
    return load().PTB_SetProfiling(int(enable))


def stage_times():
    """{stage: (ms, launches)} accumulated since the last call (profiling must be on)."""
    n = len(STAGES)
    ms = np.zeros(n)
    launches = np.zeros(n, dtype=np.uint64)
    load().PTB_StageTimes(ms.ctypes.data_as(_f64p), launches.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), n)
    return {k: (float(ms[i]), int(launches[i])) for i, k in enumerate(STAGES)}


def mle_evaluations():
    """{"lm": FP32 LM evaluations, "polish": FP32 polish evaluations, "init_final": axial pre-scan (FP32) and final
    Fisher (FP64) evaluations} counted while profiling was on (modes 6-8), and "fp64_cholesky": FP32 Cholesky solves
    redone in FP64, since the last call."""
    out = np.zeros(4, dtype=np.uint64)
    load().PTB_MleEvaluations(out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), 4)
    return {"lm": int(out[0]), "polish": int(out[1]), "init_final": int(out[2]), "fp64_cholesky": int(out[3])}


def tracking(points, max_distance):
    """Tracking: points [n, 4] (Id, Plane, X, Y) -> [n, 2] uint64 (Id, Track) in (Plane, Id) order."""
    points = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 4)
    out = np.zeros((points.shape[0], 2), dtype=np.uint64)
    if points.shape[0]:
        load().Tracking(points.ctypes.data_as(_f64p), out.ctypes.data_as(ctypes.POINTER(_u64)), points.shape[0], max_distance)
        if last_error():
            raise RuntimeError("Tracking failed: " + last_error())
    return out


def tiff_info(path):
    """(width, height, planes) of a 16-bit TIFF stack; RuntimeError on an unreadable or unsupported file."""
    w, h, z = _u64(), _u64(), _u64()
    if not load().PTB_TiffInfo(os.fsencode(path), ctypes.byref(w), ctypes.byref(h), ctypes.byref(z)):
        raise RuntimeError("PTB_TiffInfo failed: " + last_error())
    return w.value, h.value, z.value


def tiff_read(path, first=0, count=None):
    """Pages [first, first + count) of a TIFF stack as a uint16 [count, height, width] array."""
    w, h, z = tiff_info(path)
    if count is None:
        count = z - first
    out = np.empty((count, h, w), dtype=np.uint16)
    if count and load().PTB_TiffRead(os.fsencode(path), out.ctypes.data_as(_u16p), first, count) != count:
        raise RuntimeError("PTB_TiffRead failed: " + last_error())
    return out


def localization_tiff(path, thr, ratio, fit, params, capacity_doubles=None, out=None):
    """Localization of a TIFF stack on disk; returns the [n, 18] float64 rows (a view of ``out`` when given: a
    caller-owned float64 buffer, ideally pinned, whose size is the capacity)."""
    if out is not None:
        capacity_doubles = out.size
    else:
        w, h, z = tiff_info(path)
        if capacity_doubles is None:
            capacity_doubles = ((h * w) // 5 + 1) * z * COLS
        out = np.full(max(capacity_doubles, 1), -12345.0)
    params = np.ascontiguousarray(params, dtype=np.float64)
    n = load().PTB_LocalizationTiff(os.fsencode(path), out.ctypes.data_as(_f64p), capacity_doubles, thr, ratio, fit,
                                    params.ctypes.data_as(_f64p))
    if n == 0 and last_error():
        raise RuntimeError("PTB_LocalizationTiff failed: " + last_error())
    return out[:n].reshape(-1, COLS)


def graph_stats():
    """{"captured", "replayed", "direct"}: chunks of this device's engine captured into launch-chain graphs, replayed
    from them and launched directly, since the last call."""
    out = np.zeros(3, dtype=np.uint64)
    load().PTB_GraphStats(out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), 3)
    return {"captured": int(out[0]), "replayed": int(out[1]), "direct": int(out[2])}


def detect_staging_stats():
    """{"tma", "loads"}: detection launches (whole process) whose input tiles were staged by the tensor memory
    accelerator and by per-thread loads, since the last call."""
    out = np.zeros(2, dtype=np.uint64)
    load().PTB_DetectStagingStats(out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), 2)
    return {"tma": int(out[0]), "loads": int(out[1])}


def segmentation_stats():
    """{"frames", "routed", "rank_tested", "reflooded", "routed_why"}: frames segmented by this device's engines since
    the last call; of those, frames flooded again frame-wide, frames whose per-component floods needed the rank test,
    frames flooded again per component with estimated frame-wide aging because they failed it, and the nonzero counts
    of the frames flooded frame-wide by the first reason."""
    out = np.zeros(11, dtype=np.uint64)
    load().PTB_SegmentationStats(out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), 11)
    why = ("pair_list_full", "first_test_only", "no_rank_slot", "too_many_pairs", "after_fusion", "no_reflood_slot",
           "reflood_test_failed")
    return {"frames": int(out[0]), "routed": int(out[1]), "rank_tested": int(out[2]), "reflooded": int(out[3]),
            "routed_why": {k: int(out[4 + i]) for i, k in enumerate(why) if out[4 + i]}}


def spline_coefficients(psf, lam=None):
    """Cubic-spline coefficient table of a PSF volume [nz, ny, nx] (PTB_SplineCoefficients): [64, nz-1, ny-1, nx-1]."""
    psf = np.ascontiguousarray(psf, dtype=np.float64)
    nz, ny, nx = psf.shape
    out = np.zeros((64, nz - 1, ny - 1, nx - 1))
    lam_p = None
    if lam is not None:
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        lam_p = lam.ctypes.data_as(_f64p)
    n = load().PTB_SplineCoefficients(psf.ctypes.data_as(_f64p), nx, ny, nz, lam_p, out.ctypes.data_as(_f64p))
    if n == 0 or n != out.size:
        raise RuntimeError("PTB_SplineCoefficients failed: " + last_error())
    return out


def engine_pool_stats():
    """{"engines", "peak_leased"}: engines in this device's pool and the most leased at the same time."""
    out = np.zeros(2, dtype=np.uint64)
    load().PTB_EnginePoolStats(out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), 2)
    return {"engines": int(out[0]), "peak_leased": int(out[1])}


def mle_mappings():
    """Autotuned ROI mappings of modes 6-8 on this device's engines: a list of {"mode", "roi", "size_class",
    "lanes", "chunk"}."""
    out = np.zeros((64, 5), dtype=np.int32)
    n = load().PTB_MleMappings(out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), 64)
    return [dict(zip(("mode", "roi", "size_class", "lanes", "chunk"), map(int, row))) for row in out[:n]]


def fma_peak(fp64):
    """Measured FMA FLOP/s of the current device (FP64 when fp64 is true, else FP32)."""
    return load().PTB_MeasureFmaPeak(int(bool(fp64)))


def fitting_device_noalloc(d_stack_ptr, d_positions_ptr, n_points, d_output_ptr, shape, fit, params, stream_ptr=0):
    """Fit-only on device buffers without any device allocation (PTB_FittingDeviceNoAlloc); returns doubles written."""
    z, h, w = shape
    params = np.ascontiguousarray(params, dtype=np.float64)
    return load().PTB_FittingDeviceNoAlloc(ctypes.c_void_p(d_stack_ptr), ctypes.c_void_p(d_positions_ptr), n_points,
                                           ctypes.c_void_p(d_output_ptr), h, w, z, fit, params.ctypes.data_as(_f64p),
                                           ctypes.c_void_p(stream_ptr))


class Server:
    """Serving front end (PTB_ServerStart / PTB_SubmitStack / PTB_StackResult). submit() keeps references to the
    stack and the output buffer until result() returns, because the library reads and writes them asynchronously."""

    def __init__(self, slots=4, budget_bytes=0):
        if not load().PTB_ServerStart(int(slots), int(budget_bytes)):
            raise RuntimeError("PTB_ServerStart failed: " + last_error())
        self._live = {}

    def submit(self, stack, thr, ratio, fit, params, capacity_doubles=None):
        stack = _stack(stack)
        z, h, w = stack.shape
        if capacity_doubles is None:
            capacity_doubles = ((h * w) // 5 + 1) * z * COLS
        out = np.empty(max(capacity_doubles, 1))
        params = np.ascontiguousarray(params, dtype=np.float64)
        t = load().PTB_SubmitStack(stack.ctypes.data_as(_u16p), out.ctypes.data_as(_f64p), capacity_doubles, h, w, z, thr, ratio,
                                   fit, params.ctypes.data_as(_f64p))
        if t == 0:
            raise RuntimeError("PTB_SubmitStack failed: " + last_error())
        self._live[t] = (stack, out)
        return t

    def poll(self, ticket):
        return load().PTB_PollStack(ticket)

    def result(self, ticket):
        """(rows [n, 18], queueing delay s, latency s)."""
        times = np.zeros(2)
        n = load().PTB_StackResult(ticket, times.ctypes.data_as(_f64p))
        held = self._live.pop(ticket, None)
        if n < 0 or held is None:
            raise RuntimeError("PTB_StackResult failed: " + last_error())
        out = held[1]
        return out[:n].reshape(-1, COLS).copy(), float(times[0]), float(times[1])

    def fuse_stats(self):
        """{"launches", "chunks"}: fused fit launches of this server and the chunks they fitted."""
        out = np.zeros(2, dtype=np.uint64)
        load().PTB_ServerFuseStats(out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), 2)
        return {"launches": int(out[0]), "chunks": int(out[1])}

    def stop(self):
        load().PTB_ServerStop()
