"""Benchmark: localizations/s of the detect + MLE fit hot path on the 2000 x 1024 x 1024 uint16 workload.

One step = one Localization pass (wavelet -> threshold -> watershed -> per-ROI Poisson-MLE LM fit (mode 6: x, y,
sigma, photons, background) -> per-plane ordering) over the whole synthetic stack. ``value`` is measured on
device-resident frames through PTB_LocalizationDevice; ``e2e`` is the reference-facing C ABI (Localization) with
host buffers, host<->device copies inside the timed region.

The reference has no maximum-likelihood fit; its CPU arm (``--impl reference`` and ``cpu_baseline``) runs the
reference's own Localization with its 5-parameter Gaussian least-squares fit (fit mode 2: x, y, sigma, amplitude,
offset), the closest counterpart of the path, built from its sources (oracle/_ref).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--frames Z]

Under torchrun (N > 1) each rank processes its own stack of the same shape (frames shard with no exchange: weak
scaling); the max over ranks of the device time is reported.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "palmtracer-cpp_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, ROOT)

METRIC = "localizations/s (detect+MLE fit) at FP64-matched error; p50/p99 stack latency"
UNIT = "localizations/s"
WORKLOAD = "c2"
GAUSS_PARAMS = np.array([7.0, 1.3, 1.3, 0.0])
# fit_params per mode for the 7x7 workload: reference Gaussian least-squares modes (roi, sigma x, sigma y, theta) and
# the Poisson-MLE Gaussian (roi, sigma0, camera offset ADU, gain ADU/photon, max iterations, CRLB filter (0 = off))
PARAMS_BY_MODE = {0: GAUSS_PARAMS, 1: GAUSS_PARAMS, 2: GAUSS_PARAMS, 3: GAUSS_PARAMS, 4: GAUSS_PARAMS,
                  6: np.array([7.0, 1.3, 100.0, 2.0, 20.0, 0.0])}
FIT_MODE = 6
FIT_PARAMS = PARAMS_BY_MODE[FIT_MODE]
REF_FIT_MODE = 2  # the reference's own 5-parameter Gaussian fit, for the CPU arm
# Algorithmic FP32 FLOPs of one pixel of one LM evaluation of the mode-6 model (deviance, gradient, Fisher matrix):
# separable PSF and its 3 derivatives 8, mu and deviance 10, gradient terms 7, gradient 10, Fisher matrix 35
# (an FMA counts 2; a division, logarithm or reciprocal 1). Per-evaluation erf tables and the 5x5 solve are not
# counted.
FLOP_PER_PIXEL_LM = 71
# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) per frame of one launch, from ncu captures of smaller
# chunks of the same workload, scaled by the frames a benchmark launch processes (traffic grows with the frames):
# MleLmKernel<6> 127.38 MB and DetectKernel 252.41 MB over one 64-frame chunk.
LM_DRAM_BYTES_PER_FRAME = 127.38e6 / 64
DETECT_DRAM_BYTES_PER_FRAME = 252.41e6 / 64
RATIO = 0.0
PER_PLANE = 8192
# Serving mix (C5): Poisson arrivals at 20 stacks/s of square frames from {128, 256, 512, 1024, 2048}, lengths 1-500,
# half 2D Gaussian (C1 statistics, MLE mode 6, 7x7) and half astigmatic 3D (C3 statistics, MLE mode 7, 11x11).
SERVE_SIZES = [128, 256, 512, 1024, 2048]
SERVE_RATE = 20.0
SERVE_SLOTS = 4
SERVE_PER_PLANE = 2048
ASTIG = [150.0, 400.0, 0.05, 0.0, 1.3 * 160, -150.0, 400.0, -0.05, 0.0, 1.3 * 160]
MLE7_PARAMS = np.array([11.0, 160.0] + ASTIG + [100.0, 2.0, 20.0, -600.0, 600.0, 0.0])


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampler running during the timed region: started, and waited for until it has printed its first
    sample (nvidia-smi takes a fraction of a second to start), before the timed region; mark() at the start of the
    timed region, and stop() keeps the samples taken after it."""

    def __init__(self, index):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.skip = 0
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(index), "--query-gpu=" + q, "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        t0 = time.perf_counter()
        while self.proc is not None and self._lines() == 0 and time.perf_counter() - t0 < 5.0 and self.proc.poll() is None:
            time.sleep(0.02)

    def _lines(self):
        with open(self.file.name) as f:
            return sum(1 for line in f if line.endswith("\n"))

    def mark(self):
        """Samples printed so far predate the timed region."""
        if self.proc is not None:
            self.skip = self._lines()

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.file.read().splitlines()
        if len(lines) > self.skip:
            lines = lines[self.skip:]
        for line in lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.file.name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def over_ranks(dist, torch, total_ms, rows, device):
    """Whole-job figures of a multi-rank run (one process per GPU, each on its own stack): the slowest rank's timed
    milliseconds and the rows of all ranks. Every rank takes this one collective at the same point."""
    t = torch.tensor([float(total_ms), float(rows)], device=device, dtype=torch.float64)
    allt = [torch.zeros_like(t) for _ in range(dist.get_world_size())]
    dist.all_gather(allt, t)
    return max(float(x[0]) for x in allt), sum(float(x[1]) for x in allt)


def mad_threshold_gpu(lib, frame):
    import synth
    w1 = lib.wavelett(frame, 2)[0]
    return synth.mad_threshold(w1)


def reference_threshold(frame):
    """The MAD threshold of a frame's W1 plane computed by the reference build's own Wavelett (the oracle port when
    the build is absent), for the reference arm: the same value as the GPU arm's, since the planes are bit-exact."""
    import synth
    from oracle.oracle import reference, OracleLib
    lib = reference() or OracleLib()
    return synth.mad_threshold(lib.wavelett(frame, 2)[0])


def cpu_reference_rate(frames_host, thr, seconds=10.0, threads=None):
    """Reference CPU path (oracle/_ref, or the oracle port when the reference build is absent) on a bounded sample."""
    from oracle.oracle import reference, OracleLib
    lib = reference()
    kind = "reference"
    if lib is None:
        lib = OracleLib()
        kind = "port"
    cores = threads or os.cpu_count()
    lib.set_threads(cores)
    z = frames_host.shape[0]
    n0 = min(z, max(4, cores))
    t0 = time.perf_counter()
    rows = lib.localization(frames_host[:n0], thr, RATIO, REF_FIT_MODE, GAUSS_PARAMS, capacity_doubles=PER_PLANE * n0 * 18)
    dt0 = time.perf_counter() - t0
    n1 = int(min(z, max(n0, n0 * seconds / max(dt0, 1e-3))))
    if n1 > n0:
        t0 = time.perf_counter()
        rows = lib.localization(frames_host[:n1], thr, RATIO, REF_FIT_MODE, GAUSS_PARAMS, capacity_doubles=PER_PLANE * n1 * 18)
        dt0 = time.perf_counter() - t0
    else:
        n1 = n0
    return rows.shape[0] / dt0, {"kind": kind, "cores": cores,
                                 "sample": "%d of the %d frames, the reference's Localization with its fit mode %d "
                                           "(Gaussian least squares; the reference has no MLE fit)" % (n1, z, REF_FIT_MODE),
                                 "frames": n1, "seconds": dt0, "rows": int(rows.shape[0])}


def workload_runs(ptb, torch, steps=3, warmup=3):
    """The other named workloads, device-resident through PTB_LocalizationDevice, each timed with CUDA events over
    `steps` steps after `warmup`: C1 200 x 256^2 (MLE mode 6, 7x7), C3 1000 x 512^2 astigmatic (mode 7, 11x11), C4
    1500 x 512^2 with 0-1500 emitters per frame and a 25 x 25 x 121 cubic-spline PSF table (mode 8, 13x13)."""
    import spline_table
    import synth
    p8 = spline_table.fit_params(roi=13, sx=25, sy=25, sz=121, dz_nm=10.0, distortion=0.2, seed=9)
    mle8 = np.concatenate([p8[:5], [100.0, 2.0, 20.0, 0.0], p8[5:]])
    out = {}
    for name, fit, params, roi in (("c1", 6, PARAMS_BY_MODE[6], 7), ("c3", 7, MLE7_PARAMS, 11), ("c4", 8, mle8, 13)):
        d_in, _ = synth.stack_cuda(name, seed=4242)
        z, h, w = d_in.shape
        thr = mad_threshold_gpu(ptb, d_in[0].cpu().numpy().view(np.uint16))
        cap = PER_PLANE * z * 18
        d_out = torch.empty(cap, dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream()

        def step():
            return ptb.localization_device(d_in.data_ptr(), d_out.data_ptr(), cap, (z, h, w), thr, RATIO, fit, params,
                                           stream.cuda_stream)

        for _ in range(warmup):
            n = step()
        torch.cuda.synchronize()
        ptb.segmentation_stats()  # counts of the timed steps only
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            n = step()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        seg = ptb.segmentation_stats()
        # stage breakdown of one more (untimed) pass, chunks serialised
        ptb.set_profiling(1)
        ptb.stage_times()
        step()
        torch.cuda.synchronize()
        stages = ptb.stage_times()
        ptb.set_profiling(0)
        rows = n // 18
        out[name] = {"frames": z, "height": h, "width": w, "fit_mode": fit, "roi": roi, "localizations_per_step": int(rows),
                     "ms_per_step": ms, "localizations_per_s": rows / (ms / 1000.0), "frames_per_s": z / (ms / 1000.0),
                     "segmentation": seg, "stage_ms": {k: round(v[0], 3) for k, v in stages.items()}}
        del d_in, d_out
        torch.cuda.empty_cache()
    return out


TRACK_DISTANCE = 5.0  # maxDistance of the reference's tracking tests (Tests_CPU/test_tr_Tracks.cpp:262)


def tracking_run(ptb, torch, d_rows, n_rows, sample_planes=200):
    """Tracking (the reference's Tracking export) of the benchmark's own localization table: device-resident through
    PTB_TrackingDevice (CUDA events around the call, which synchronizes once to size its scratch), end to end through
    the host Tracking export, and the reference CPU build on the table's first `sample_planes` planes with all host
    threads; the GPU result on that sample is compared bit for bit with the reference's."""
    from oracle.oracle import reference, OracleLib
    rows = d_rows[: n_rows * 18].view(n_rows, 18)
    pts = rows[:, [0, 1, 4, 5]].contiguous()
    n = pts.shape[0]
    out = torch.empty((n, 2), dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream()
    L = ptb.load()
    dev_ms = []
    for i in range(4):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        if L.PTB_TrackingDevice(pts.data_ptr(), out.data_ptr(), n, TRACK_DISTANCE, stream.cuda_stream) != 2 * n:
            raise RuntimeError("PTB_TrackingDevice failed: " + ptb.last_error())
        e1.record(stream)
        e1.synchronize()
        if i:
            dev_ms.append(e0.elapsed_time(e1))
    host_pts = pts.cpu().numpy()
    e2e_s = []
    for i in range(3):
        t0 = time.perf_counter()
        got = ptb.tracking(host_pts, TRACK_DISTANCE)
        if i:
            e2e_s.append(time.perf_counter() - t0)
    tracks = int(got[:, 1].max()) if n else 0
    cpu = reference()
    kind = "reference"
    if cpu is None:
        cpu, kind = OracleLib(), "port"
    cores = os.cpu_count()
    cpu.set_threads(cores)
    sample = host_pts[host_pts[:, 1] <= sample_planes]
    t0 = time.perf_counter()
    want = cpu.tracking(sample, TRACK_DISTANCE)
    cpu_s = time.perf_counter() - t0
    same = bool(np.array_equal(ptb.tracking(sample, TRACK_DISTANCE), want))
    dev = float(np.median(dev_ms)) / 1000.0
    return {"workload": "the benchmark's %d localizations over %d planes, maxDistance %.1f px (%d tracks)"
                        % (n, int(host_pts[:, 1].max()), TRACK_DISTANCE, tracks),
            "unit": "points/s", "device": {"value": n / dev, "ms": dev * 1000.0},
            "e2e": {"value": n / float(np.median(e2e_s)), "ms": float(np.median(e2e_s)) * 1000.0,
                    "h2d_bytes": int(n * 32), "d2h_bytes": int(n * 16)},
            "cpu_baseline": {"value": sample.shape[0] / cpu_s, "kind": kind, "cores": cores,
                             "sample": "the first %d planes (%d points)" % (sample_planes, sample.shape[0]),
                             "seconds": cpu_s},
            "parity_on_sample": same}


def serving_run(ptb, torch, n_req, seed=2026):
    """C5 serving mix through PTB_ServerStart / PTB_SubmitStack / PTB_StackResult: a Poisson-arrival run at
    SERVE_RATE, a saturated run (every request submitted at once) and the plain one-call-per-frame form on a
    bounded sample of the same frames. Latencies are measured by the library from submission to completion."""
    import synth
    rng = np.random.default_rng(seed)
    sizes = rng.choice(SERVE_SIZES, n_req)
    kinds = rng.integers(0, 2, n_req)
    lengths = rng.integers(1, 501, n_req)
    arrivals = np.cumsum(rng.exponential(1.0 / SERVE_RATE, n_req))
    base = {}
    for size, kind in sorted(set(zip(sizes.tolist(), kinds.tolist()))):
        frames = int(lengths[(sizes == size) & (kinds == kind)].max())
        d, _ = synth.stack_cuda("c1" if kind == 0 else "c3", frames=frames, seed=seed + 7 * size + kind, size=(size, size))
        host = torch.empty(d.shape, dtype=torch.int16, pin_memory=True)
        host.copy_(d)
        del d
        arr = host.numpy().view(np.uint16)
        base[(size, kind)] = (host, arr, mad_threshold_gpu(ptb, arr[0]))
    torch.cuda.empty_cache()
    fit_of = {0: (6, PARAMS_BY_MODE[6]), 1: (7, MLE7_PARAMS)}
    server = ptb.Server(slots=SERVE_SLOTS)
    fused = None

    def submit(i):
        _, arr, thr = base[(int(sizes[i]), int(kinds[i]))]
        fit, params = fit_of[int(kinds[i])]
        return server.submit(arr[:int(lengths[i])], thr, RATIO, fit, params, capacity_doubles=SERVE_PER_PLANE * int(lengths[i]) * 18)

    def collect(tickets):
        rows, lat = 0, []
        for t in tickets:
            r, _, latency = server.result(t)
            rows += r.shape[0]
            lat.append(latency * 1000.0)
        return rows, np.array(lat)

    try:
        for kind in (0, 1):  # warm-up: one small stack per model
            i = int(np.argmin(np.where(kinds == kind, sizes * lengths, 1 << 40)))
            collect([submit(i)])
        t0 = time.perf_counter()
        tickets = []
        for i in range(n_req):
            wait = t0 + arrivals[i] - time.perf_counter()
            if wait > 0:
                time.sleep(wait)
            tickets.append(submit(i))
        rows, lat = collect(tickets)
        poisson_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        rows_sat, lat_sat = collect([submit(i) for i in range(n_req)])
        sat_s = time.perf_counter() - t0
        fused = server.fuse_stats()
    finally:
        server.stop()
    # the same saturated run with every slot fitting its own chunks (no fused launches), for comparison
    os.environ["PTB_FUSE_FITS"] = "0"
    try:
        server = ptb.Server(slots=SERVE_SLOTS)
        try:
            for kind in (0, 1):
                i = int(np.argmin(np.where(kinds == kind, sizes * lengths, 1 << 40)))
                collect([submit(i)])
            t0 = time.perf_counter()
            rows_unf, lat_unf = collect([submit(i) for i in range(n_req)])
            unf_s = time.perf_counter() - t0
        finally:
            server.stop()
    finally:
        del os.environ["PTB_FUSE_FITS"]
    # plain form: one Localization call per frame, on the first frames of the same requests (bounded sample)
    plain_rows, plain_frames, plain_lat, t_start = 0, 0, [], time.perf_counter()
    for i in range(n_req):
        _, arr, thr = base[(int(sizes[i]), int(kinds[i]))]
        fit, params = fit_of[int(kinds[i])]
        for z in range(min(int(lengths[i]), 8)):
            t1 = time.perf_counter()
            r = ptb.localization(arr[z:z + 1], thr, RATIO, fit, params, capacity_doubles=SERVE_PER_PLANE * 18)
            plain_lat.append((time.perf_counter() - t1) * 1000.0)
            plain_rows += r.shape[0]
            plain_frames += 1
        if time.perf_counter() - t_start > 8.0:
            break
    plain_s = time.perf_counter() - t_start
    frames_total = int(lengths.sum())
    # pixels copied host -> device for the whole mix: with the GPU faster than the link, this is what bounds it
    in_bytes = int((lengths.astype(np.int64) * sizes.astype(np.int64) ** 2 * 2).sum())
    return {
        "workload": "C5: %d stacks, Poisson arrivals at %.0f stacks/s, square frames of %s px, 1-500 frames (%d in all), "
                    "half 2D Gaussian (MLE mode 6, 7x7), half astigmatic 3D (MLE mode 7, 11x11); %d server slots"
                    % (n_req, SERVE_RATE, "/".join(str(s) for s in SERVE_SIZES), frames_total, SERVE_SLOTS),
        "input_bytes": in_bytes,
        "poisson": {"localizations_per_s": rows / poisson_s, "frames_per_s": frames_total / poisson_s, "seconds": poisson_s,
                    "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))}},
        "saturated": {"localizations_per_s": rows_sat / sat_s, "frames_per_s": frames_total / sat_s, "seconds": sat_s,
                      "h2d_gbs": in_bytes / sat_s / 1e9,
                      "latency_ms": {"p50": float(np.percentile(lat_sat, 50)), "p99": float(np.percentile(lat_sat, 99))},
                      "fused_fit_launches": fused},
        "saturated_unfused": {"localizations_per_s": rows_unf / unf_s, "seconds": unf_s,
                              "latency_ms": {"p50": float(np.percentile(lat_unf, 50)), "p99": float(np.percentile(lat_unf, 99))}},
        "plain_per_frame": {"localizations_per_s": plain_rows / plain_s, "frames_per_s": plain_frames / plain_s,
                            "sample_frames": plain_frames,
                            "call_latency_ms": {"p50": float(np.percentile(plain_lat, 50)), "p99": float(np.percentile(plain_lat, 99))}},
        "localizations": int(rows),
    }


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def parity_run(ptb, d_in, thr, n_cand=16, n_mle=4):
    """Parity of the benchmark's own frames, outside the timed region: the candidate rows (fit 0: Id, Plane, Index,
    X, Y, SegIntensity, Surface of every candidate) of the first `n_cand` frames against the reference build, bit
    for bit, and the error table of the benchmark fit (mode 6) on the first `n_mle` frames against the FP64 oracle
    (median / p99 / max of |GPU - oracle| per quantity; x, y, sigma in px, photons and background relative)."""
    from compare import match_rows, C_X, C_Y, C_SX, C_OFF
    from oracle.oracle import reference, OracleLib
    host = d_in[:n_cand].cpu().numpy().view(np.uint16)
    cap = PER_PLANE * n_cand * 18
    ref = reference()
    kind = "reference build" if ref is not None else "oracle port"
    ref = ref or OracleLib()
    ref.set_threads(os.cpu_count())
    a = ptb.localization(host, thr, RATIO, 0, GAUSS_PARAMS, capacity_doubles=cap)
    b = ref.localization(host, thr, RATIO, 0, GAUSS_PARAMS, capacity_doubles=cap)
    same = bool(a.shape == b.shape and np.array_equal(a, b))
    orc = OracleLib()
    orc.set_threads(os.cpu_count())
    m = host[:n_mle]
    ga = ptb.localization(m, thr, RATIO, FIT_MODE, FIT_PARAMS, capacity_doubles=PER_PLANE * n_mle * 18)
    gb = orc.localization(m, thr, RATIO, FIT_MODE, FIT_PARAMS, capacity_doubles=PER_PLANE * n_mle * 18)
    out = {"candidates_equal": same, "candidate_frames": n_cand, "candidates": int(a.shape[0]), "candidates_against": kind,
           "mle_frames": n_mle, "mle_fits": int(ga.shape[0]), "mle_against": "FP64 oracle (oracle/pt_oracle.cpp)"}
    bad, _, pairs = match_rows(ga, gb, atol=1e9, rtol=0, keys=(C_X, C_Y))
    if pairs is None or bad:
        out["mle_errors"] = None
        out["mle_unmatched_rows"] = int(bad)
        return out
    e = gb[pairs]
    both = (ga[:, C_SX] >= 0) & (e[:, C_SX] >= 0)
    tol = {"x": ("abs", C_X, 1e-3), "y": ("abs", C_Y, 1e-3), "photons": ("rel", 7, 1e-4), "background": ("rel", C_OFF, 1e-4),
           "sigma": ("abs", C_SX, 1e-4)}
    beyond = np.zeros(len(ga), dtype=bool)
    errs = {}
    for key, (kind_, c, t) in tol.items():
        d = np.abs(ga[:, c] - e[:, c])
        if kind_ == "rel":
            d = d / np.abs(e[:, c])
        d = d[both]
        beyond[both] |= d > t
        errs[key] = {"kind": kind_, "tol": t, "median": float(np.median(d)), "p99": float(np.percentile(d, 99)),
                     "max": float(np.max(d))}
    out["mle_errors"] = errs
    out["mle_fits_compared"] = int(both.sum())
    out["mle_beyond_tolerance"] = int(beyond.sum())
    out["mle_status_flips"] = int(np.sum((ga[:, C_SX] >= 0) != (e[:, C_SX] >= 0)))
    return out


def same_work_run(ptb, torch, d_in, thr, frames, h, w, steps=3):
    """The reference arm's own fit (mode 2: Gaussian least squares, FP64, the reference's operation order) on the
    benchmark stack: device-resident and end to end through Localization with pinned host buffers. Beside the
    reference arm's number this is a same-work ratio."""
    cap = PER_PLANE * frames * 18
    d_out = torch.empty(cap, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()

    def step():
        return ptb.localization_device(d_in.data_ptr(), d_out.data_ptr(), cap, (frames, h, w), thr, RATIO, REF_FIT_MODE,
                                       GAUSS_PARAMS, stream.cuda_stream)

    n = step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        n = step()
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    rows = n // 18
    del d_out
    host_in = torch.empty((frames, h, w), dtype=torch.int16, pin_memory=True)
    host_in.copy_(d_in)
    host_np = host_in.numpy().view(np.uint16)
    host_out = torch.empty(cap, dtype=torch.float64, pin_memory=True).numpy()
    e2e = []
    for i in range(steps + 1):
        t0 = time.perf_counter()
        k = ptb.localization_raw(host_np, host_out, thr, RATIO, REF_FIT_MODE, GAUSS_PARAMS)
        if i:
            e2e.append(time.perf_counter() - t0)
    del host_in, host_out
    e2e_s = float(np.median(e2e))
    return {"fit_mode": REF_FIT_MODE, "fit": "Gaussian least squares (x, y, sigma, amplitude, offset), FP64, in the "
                                             "reference's order of operations", "localizations_per_step": int(rows),
            "device": {"ms_per_step": ms, "localizations_per_s": rows / (ms / 1000.0)},
            "e2e": {"ms_per_step": e2e_s * 1000.0, "localizations_per_s": (k // 18) / e2e_s}}


def plain_per_frame_run(ptb, host_frames, thr, seconds=6.0):
    """The plain drop-in form on the benchmark's own frames: one Localization call per 1024 x 1024 frame with
    pageable host buffers, as a front end that hands over frame after frame would call it; call latency p50 / p99 and
    the throughput of the calls (a bounded sample)."""
    lat, rows, t_start = [], [], time.perf_counter()
    for z in range(host_frames.shape[0]):
        frame = np.ascontiguousarray(host_frames[z:z + 1])
        t1 = time.perf_counter()
        r = ptb.localization(frame, thr, RATIO, FIT_MODE, FIT_PARAMS, capacity_doubles=PER_PLANE * 18)
        lat.append(time.perf_counter() - t1)
        rows.append(r.shape[0])
        if time.perf_counter() - t_start > seconds and z >= 20:
            break
    lat = np.array(lat[2:])  # the first two calls launch the chain directly, then capture its graph
    total = float(lat.sum())
    per_frame = float(np.mean(rows[2:]))
    p99 = float(np.percentile(lat, 99))
    return {"frames": int(len(lat)), "localizations_per_s": per_frame * len(lat) / total,
            "call_latency_ms": {"p50": float(np.percentile(lat, 50)) * 1000.0, "p99": p99 * 1000.0},
            # throughput of a front end that budgets every call at the p99 latency
            "p99_bounded_localizations_per_s": per_frame / p99}


def main():
    global FIT_MODE, FIT_PARAMS
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", type=int, default=0, help="fit arithmetic (PTB_SetFitPrecision)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--fit", type=int, default=None, help="fit mode (default: %d)" % FIT_MODE)
    ap.add_argument("--no-serving", action="store_true", help="skip the C5 serving mix")
    ap.add_argument("--no-tracking", action="store_true", help="skip tracking the benchmark's localizations")
    ap.add_argument("--no-workloads", action="store_true", help="skip the C1, C3 and C4 workloads")
    ap.add_argument("--serve-requests", type=int, default=40)
    ap.add_argument("--no-parity", action="store_true", help="skip the parity check of the benchmark's own frames")
    ap.add_argument("--no-pageable", action="store_true", help="skip the end-to-end run from pageable host memory")
    args = ap.parse_args()
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=180))
    torch.cuda.set_device(local)
    import synth

    if args.fit is not None:
        FIT_MODE = args.fit
        FIT_PARAMS = PARAMS_BY_MODE[FIT_MODE]
    frames = args.frames or synth.SHAPES[WORKLOAD][0]
    h, w = synth.SHAPES[WORKLOAD][1:]
    # one config for both arms (the reference has no MLE fit: its arm runs its own least-squares mode 2)
    config = {"workload": "c2: %d frames of %dx%d uint16, ~2684 emitters/frame, 7x7 ROI, per-plane capacity %d"
                          % (frames, h, w, PER_PLANE),
              "frames": frames, "height": h, "width": w, "roi": 7, "watershed_ratio": RATIO,
              "fit_modes": {"this_library": FIT_MODE, "reference_arm": REF_FIT_MODE},
              "l2": "inputs (4.2 GB) larger than L2", "parallelism": "frames sharded, no exchange" if world > 1 else "single GPU"}

    if args.impl == "reference":
        if rank != 0:
            if world > 1:
                dist.destroy_process_group()
            return
        # the frames come from the same seeded GPU generator as the other arm's; nothing of this library runs here
        d, _ = synth.stack_cuda(WORKLOAD, frames=min(frames, 256), seed=1000)
        host = d.cpu().numpy().view(np.uint16)
        thr = reference_threshold(host[0])
        del d
        torch.cuda.empty_cache()
        rates = []
        info = None
        for i in range(args.warmup + args.steps):
            r, info = cpu_reference_rate(host, thr, seconds=8.0)
            if i >= args.warmup:
                rates.append(r)
        v = float(np.median(rates))
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": config,
                "cpu_baseline": {"value": v, "unit": UNIT, "cores": info["cores"], "kind": info["kind"], "sample": info["sample"],
                                 "cpu_model": cpu_model()},
                "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return

    import ptb
    ptb.set_fit_precision(args.precision)
    d_in, em = synth.stack_cuda(WORKLOAD, frames=frames, seed=1000 + rank)
    torch.cuda.synchronize()
    thr = mad_threshold_gpu(ptb, d_in[0].cpu().numpy().view(np.uint16))
    cap = PER_PLANE * frames * 18
    d_out = torch.empty(cap, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()

    def step():
        return ptb.localization_device(d_in.data_ptr(), d_out.data_ptr(), cap, (frames, h, w), thr, RATIO, FIT_MODE, FIT_PARAMS,
                                       stream.cuda_stream)

    for _ in range(args.warmup):
        n = step()
    if n == 0:
        raise RuntimeError("no localizations: " + ptb.last_error())
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = Clocks(local)
    ptb.segmentation_stats()
    launches0 = ptb.launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    counts = []
    torch.cuda.synchronize()
    clocks.mark()
    for e0, e1 in ev:
        e0.record(stream)
        counts.append(step())
        e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    launches = (ptb.launch_count() - launches0) // args.steps
    seg = ptb.segmentation_stats()
    step_ms = np.array([a.elapsed_time(b) for a, b in ev])
    rows = counts[-1] // 18
    total_ms = float(step_ms.sum())
    if world > 1:
        total_ms, rows_all = over_ranks(dist, torch, total_ms, rows, "cuda")
    else:
        rows_all = float(rows)
    value = rows_all * args.steps / (total_ms / 1000.0)
    # the ROI mapping the autotuner chose for the timed steps (lanes per ROI 1: a thread per ROI; 32: a warp)
    mapping = [m for m in ptb.mle_mappings() if m["mode"] == FIT_MODE]
    lanes_txt = ", ".join(sorted({"%d lanes, chunk %d" % (m["lanes"], m["chunk"]) for m in mapping})) or "not tuned"

    # stage breakdown of one more (untimed) pass, with the MLE phases timed by CUDA events on the library's stream
    ptb.set_profiling(1)
    ptb.stage_times()
    ptb.mle_evaluations()
    step()
    torch.cuda.synchronize()
    stages = ptb.stage_times()
    evals = ptb.mle_evaluations()
    ptb.set_profiling(0)
    peak, peak_kind = peaks()
    det_ms, det_l = stages["detect"]
    det_bytes = 2.0 * h * w * frames
    det_achieved = det_bytes / (det_ms / 1000.0) / 1e9 if det_ms > 0 else None
    frames_per_launch = frames / max(det_l, 1)
    detect_roofline = {"kernel": "DetectKernel (wavelet + threshold + seeds)", "bound": "hbm", "achieved": det_achieved,
                       "peak": peak, "unit": "GB/s", "frac": (det_achieved / peak) if det_achieved else None,
                       "traffic": DETECT_DRAM_BYTES_PER_FRAME * frames_per_launch, "traffic_unit": "bytes per launch (ncu, scaled)",
                       "algorithmic_bytes_per_launch": det_bytes / max(det_l, 1), "launches": det_l,
                       "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                       "why_this_kernel": "largest share of device time in the ncu launch list of this command"}
    # the FP32 roofline of the fit's largest kernel, the second largest share
    fit_roofline = None
    if FIT_MODE == 6 and stages["fit_lm"][0] > 0:
        fp32_peak = ptb.fma_peak(False) / 1e12
        lm_ms = stages["fit_lm"][0]
        flops = FLOP_PER_PIXEL_LM * 49 * evals["lm"]
        achieved = flops / (lm_ms / 1000.0) / 1e12
        fit_roofline = {"kernel": "MleLmKernel<6> (persistent FP32 LM; ROI mapping %s)" % lanes_txt, "bound": "fp32",
                    "achieved": achieved,
                    "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                    "traffic": LM_DRAM_BYTES_PER_FRAME * frames / max(1, stages["fit_lm"][1]),
                    "traffic_unit": "bytes per launch (ncu, scaled)",
                    "algorithmic_flops_per_launch": flops / max(1, stages["fit_lm"][1]), "launches": stages["fit_lm"][1],
                    "flop_per_pixel_evaluation": FLOP_PER_PIXEL_LM, "evaluations": evals,
                    "peak_source": "measured in this run (PTB_MeasureFmaPeak FP32 FMA chains)"}
    roofline = detect_roofline
    roofline["stage_ms"] = {k: round(v[0], 3) for k, v in stages.items()}
    roofline["stage_launches"] = {k: v[1] for k, v in stages.items()}

    parity = None
    if rank == 0 and not args.no_parity:
        parity = parity_run(ptb, d_in, thr)
        parity["frames_flooded_again_frame_wide"] = {"timed_steps": seg["routed"], "frames_segmented": seg["frames"],
                                                     "frames_given_the_rank_test": seg["rank_tested"]}

    # end to end through the reference-facing C ABI with host buffers
    host_in = torch.empty((frames, h, w), dtype=torch.int16, pin_memory=True)
    host_in.copy_(d_in)
    host_np = host_in.numpy().view(np.uint16)
    h2d_bytes = int(host_np.nbytes)
    host_out = torch.empty(cap, dtype=torch.float64, pin_memory=True).numpy()
    e2e_ms = []
    n_e2e = 0
    # two untimed calls (the second captures the chunks' launch graphs), then at least five timed ones; the value is
    # taken at the median call, since the host and its PCIe links are shared with other jobs (the mean and every
    # call's time are reported beside it)
    e2e_warm = 2
    for i in range(0 if args.no_e2e else e2e_warm + max(5, args.steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        n_e2e = ptb.localization_raw(host_np, host_out, thr, RATIO, FIT_MODE, FIT_PARAMS)
        torch.cuda.synchronize()
        if i >= e2e_warm:
            e2e_ms.append((time.perf_counter() - t0) * 1000.0)
    e2e_value = (n_e2e // 18) / (float(np.median(e2e_ms)) / 1000.0) if e2e_ms else None
    # the link's own host -> device rate from pinned memory (one 1 GiB copy of the same buffer, best of 3): the
    # roofline of the e2e number
    link_gbs = None
    if e2e_ms:
        part = host_in.view(-1)[: min(host_in.numel(), 1 << 29)]
        dev = torch.empty_like(part, device="cuda")
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        best = 1e30
        for _ in range(3):
            ev0.record()
            dev.copy_(part, non_blocking=True)
            ev1.record()
            ev1.synchronize()
            best = min(best, ev0.elapsed_time(ev1))
        link_gbs = part.numel() * 2 / (best / 1000.0) / 1e9
        del dev

    # the same call with a pageable numpy copy of the input and pageable output, as most front ends pass them
    e2e_pageable = None
    if e2e_ms and rank == 0 and not args.no_pageable:
        page_in = np.array(host_np, copy=True)
        page_out = np.empty(cap, dtype=np.float64)
        pg = []
        for i in range(1 + max(3, min(args.steps, 5))):
            t0 = time.perf_counter()
            n_pg = ptb.localization_raw(page_in, page_out, thr, RATIO, FIT_MODE, FIT_PARAMS)
            if i:
                pg.append((time.perf_counter() - t0) * 1000.0)
        e2e_pageable = {"value": (n_pg // 18) / (float(np.median(pg)) / 1000.0), "unit": UNIT,
                        "ms_per_step": float(np.median(pg)), "ms_each": [round(t, 3) for t in pg],
                        "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": int(n_pg * 8)}
        del page_in, page_out

    same_work = None
    plain_c2 = None
    if rank == 0 and world == 1 and not args.no_workloads:
        same_work = same_work_run(ptb, torch, d_in, thr, frames, h, w)
        plain_c2 = plain_per_frame_run(ptb, host_np[:400], thr)
        plain_c2["batched_e2e_over_plain"] = e2e_value / plain_c2["localizations_per_s"] if e2e_value else None
        plain_c2["batched_device_over_plain"] = value / plain_c2["localizations_per_s"]
        plain_c2["batched_e2e_over_plain_p99_bounded"] = (e2e_value / plain_c2["p99_bounded_localizations_per_s"]
                                                         if e2e_value else None)

    tracking = None
    if rank == 0 and world == 1 and not args.no_tracking:
        tracking = tracking_run(ptb, torch, d_out, int(rows))
    workloads = None
    if rank == 0 and world == 1 and not args.no_workloads:
        workloads = workload_runs(ptb, torch)

    serving = None
    if rank == 0 and world == 1 and not args.no_serving:
        del host_in, host_np, host_out
        serving = serving_run(ptb, torch, args.serve_requests)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sample = d_in[: min(frames, 512)].cpu().numpy().view(np.uint16)
        v, info = cpu_reference_rate(sample, thr, seconds=10.0)
        v1, info1 = cpu_reference_rate(sample, thr, seconds=5.0, threads=1)
        cpu = {"value": v, "unit": UNIT, "cores": info["cores"], "kind": info["kind"], "sample": info["sample"],
               "cpu_model": cpu_model(), "single_thread": {"value": v1, "cores": 1, "sample": info1["sample"]}}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": ("f32 (axial pre-scan, LM and Newton polish; f64 Cholesky fallback, Fisher information, CRLB)" if FIT_MODE >= 6 else
                          "f64" if args.precision != 1 else "f32 (f64 re-fit)"),
                "data": "synthetic (seeded, generated on the GPU; no public dataset)",
                "config": config, "fit_precision": args.precision, "mle_mapping": mapping,
                "frames_per_s": frames * world * args.steps / (total_ms / 1000.0),
                "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99))},
                "localizations_per_step": int(rows_all), "roofline": roofline, "fit_roofline": fit_roofline,
                "cpu_baseline": cpu,
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d_bytes,
                        "d2h_bytes_per_step": int(n_e2e * 8), "ms_per_step": float(np.median(e2e_ms)) if e2e_ms else None,
                        "ms_mean": float(np.mean(e2e_ms)) if e2e_ms else None, "ms_each": [round(t, 3) for t in e2e_ms],
                        # host -> device rate over the median call (the frames cross PCIe once; the link is the e2e bound)
                        "h2d_gbs": h2d_bytes / (float(np.median(e2e_ms)) / 1000.0) / 1e9 if e2e_ms else None,
                        "h2d_link_gbs": link_gbs},
                "e2e_pageable": e2e_pageable, "parity": parity,
                "gpu_launches": int(launches), "clocks": clk, "serving": serving, "tracking": tracking,
                "workloads": dict(workloads or {}, c2_mode2=same_work, plain_per_frame_c2=plain_c2)}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
