"""The detection kernel runs on the CPU under AddressSanitizer against the oracle's W1, threshold and local maxima.

tests/emu/shim.h runs every CUDA thread of a block as a host thread and tests/emu/detect_driver.cpp runs DetectKernel
(detect.cu, 128 x 28 tiles) on a stack of frames, each device array its own heap allocation, so that an out-of-bounds
access anywhere in it aborts. Its code bytes, the W1 of domain pixels, the domain and seed lists and the per-frame
counts must equal the oracle's W1 (ATrous.cpp:23-80 restated in oracle/pt_oracle.cpp) thresholded strictly and above
1e-8, with seeds at the pixels not below any 3 x 3 neighbour (Segmentation2D.cpp:294-333, the frame surrounded by
zeros). The shapes cover ragged last tiles in both directions, widths that do and do not allow the 16-byte staging
loads, the widths that are multiples of 8 through the TMA staging path (its box copy emulated with the same zero fill,
then the kernel's own replication of the nearest in-frame rows and columns), frames smaller than the halo and several
frames; the stacks are full-range noise (sums up to the 2^32 limit
of the level-2 taps) and C2 frames; threshold 0 makes most pixels domain.
"""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "palmtracer-cpp_b200", "csrc")
CUDA_INCLUDE = "/usr/local/cuda/include"


def _kernels_only(src, cuts):
    """Drops the host functions (they use the <<< >>> launch syntax) between each pair of markers."""
    for start, stop in cuts:
        a = src.index(start)
        b = src.index(stop, a)
        src = src[:a] + src[b:]
    src = src.replace('#include "pt_common.cuh"', '#include "%s"' % os.path.join(CSRC, "pt_common.cuh"))
    # dynamic shared memory: a static buffer (blocks run one at a time)
    return re.sub(r'extern __shared__ (__align__\(\d+\) )?([\w ]+?) (\w+)\[\];', r'static \1\2 \3[262144];', src)


@pytest.fixture(scope="module")
def emulator(tmp_path_factory):
    if shutil.which("g++") is None or not os.path.exists(os.path.join(CUDA_INCLUDE, "cuda_runtime.h")):
        pytest.skip("g++ or the CUDA headers are missing")
    d = tmp_path_factory.mktemp("emu_detect")
    cuts = [("bool ConfigureSmem()", "}  // namespace\n"), ("long long ThresholdFixed(", "}  // namespace ptb")]
    open(d / "detect_emu.inc", "w").write(_kernels_only(open(os.path.join(CSRC, "detect.cu")).read(), cuts))
    exe = d / "emu_detect"
    cmd = ["g++", "-std=c++20", "-O2", "-g", "-fsanitize=address", "-pthread", "-Wno-attributes",
           "-I" + CUDA_INCLUDE, "-I" + str(d), "-I" + os.path.join(HERE, "emu"),
           os.path.join(HERE, "emu", "detect_driver.cpp"), "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return exe


def _run(exe, stack, thr_fixed):
    b, h, w = stack.shape
    d = os.path.dirname(str(exe))
    inp, out = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
    with open(inp, "wb") as f:
        np.array([h, w, b], dtype=np.int32).tofile(f)
        np.array([thr_fixed], dtype=np.int64).tofile(f)
        np.ascontiguousarray(stack, dtype=np.uint16).tofile(f)
    r = subprocess.run([str(exe), inp, out], capture_output=True, text=True,
                       env=dict(os.environ, ASAN_OPTIONS="detect_leaks=0"), timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    raw = np.fromfile(out, dtype=np.uint8)
    p = b * h * w
    head = raw[:12].view(np.uint32)
    o = 12
    fdom = raw[o:o + 4 * b].view(np.uint32); o += 4 * b
    fseed = raw[o:o + 4 * b].view(np.uint32); o += 4 * b
    code = raw[o:o + p]; o += p
    w1 = raw[o:o + 4 * p].view(np.uint32); o += 4 * p
    lists = raw[o:].view(np.uint32)
    nd, ns = int(head[0]), int(head[1])
    assert lists.size == nd + ns
    return {"overflow": int(head[2]), "fdom": fdom.copy(), "fseed": fseed.copy(), "code": code.copy(),
            "w1": np.where((code & 1) != 0, w1, 0), "dom": lists[:nd].copy(), "seeds": lists[nd:].copy()}


def _expected(orc, stack, thr_fixed):
    code = []
    w1s = []
    for fr in stack:
        w1 = orc.planes(fr)[1] * 65536
        assert np.array_equal(w1, np.round(w1))  # W1 is an exact multiple of 2^-16
        w1 = w1.astype(np.int64)
        dom = (w1 > thr_fixed) & (w1 > 0)  # the thresholded potential above 1e-8
        pad = np.pad(w1, 1)
        h, w = w1.shape
        mx = np.max([pad[1 + dy:1 + dy + h, 1 + dx:1 + dx + w] for dy in (-1, 0, 1) for dx in (-1, 0, 1)], axis=0)
        seed = dom & (w1 >= mx)
        code.append(dom.astype(np.uint8) | (seed.astype(np.uint8) << 1))
        w1s.append(np.where(dom, w1, 0))
    return np.stack(code).reshape(-1), np.stack(w1s).reshape(-1).astype(np.uint32)


def _thresholds(orc, stack):
    import synth
    base = synth.mad_threshold(orc.planes(stack[0])[1])
    return int(np.floor(base * 65536)), int(np.floor(0.3 * base * 65536)), 0, -5


CASES = [  # (H, W, frames, seed)
    (130, 112, 2, 1),   # a last tile row of 18 rows, one tile column short of full
    (300, 250, 1, 2),   # width not a multiple of 8: clamped 2-byte staging loads everywhere
    (60, 400, 2, 3),    # width a multiple of 8: TMA staging (on the GPU), border tiles replicate edges
    (16, 336, 1, 4),    # one short tile row
    (29, 129, 1, 5),    # one row and one column past full tiles
    (3, 17, 2, 6),      # frames smaller than the 7-pixel halo in both directions
    (257, 113, 1, 7),   # a last tile row of 5 rows
    (5, 8, 2, 8),       # the narrowest frames the TMA describes: its box reaches past every side
]


@pytest.mark.parametrize("case", CASES, ids=["x".join(map(str, c[:3])) for c in CASES])
def test_emulated_detection_matches_oracle(emulator, orc, case):
    import synth
    h, w, b, seed = case
    rng = np.random.default_rng(seed)
    # full-range noise (intermediate sums up to the 2^32 limit of V2) on every shape, C2 frames where they fit
    stacks = [rng.integers(0, 65536, size=(b, h, w), dtype=np.uint16)]
    if min(h, w) >= 64:
        stacks.append(synth.stack("c2", frames=b, seed=seed, size=(h, w))[0])
    for stack, thr in ((st, t) for st in stacks for t in _thresholds(orc, st)):
        want_code, want_w1 = _expected(orc, stack, thr)
        g = _run(emulator, stack, thr)
        assert g["overflow"] == 0
        assert np.array_equal(g["code"], want_code), (thr, int(np.sum(g["code"] != want_code)))
        assert np.array_equal(g["w1"], want_w1), thr
        assert np.array_equal(g["dom"], np.flatnonzero(want_code & 1).astype(np.uint32)), thr
        assert np.array_equal(g["seeds"], np.flatnonzero(want_code & 2).astype(np.uint32)), thr
        assert np.array_equal(g["fdom"], (want_code.reshape(b, -1) & 1).sum(axis=1)), thr
        assert np.array_equal(g["fseed"], ((want_code.reshape(b, -1) & 2) != 0).sum(axis=1)), thr
