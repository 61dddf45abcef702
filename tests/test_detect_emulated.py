"""The two detection kernels run on the CPU under AddressSanitizer: same outputs, and the oracle's W1 and threshold.

tests/emu/shim.h runs every CUDA thread of a block as a host thread and tests/emu/detect_driver.cpp runs one detection
kernel on a stack of frames, each device array its own heap allocation: DetectKernel (detect.cu, 128 x 28 tiles) and
DetectStream (detect_stream.cu, a warp per 112-column strip sweeping 128 rows). Both must write the same code bytes,
the same W1 on domain pixels, the same domain and seed lists and per-frame counts, and these must equal the oracle's
W1 (ATrous.cpp:23-80 restated in oracle/pt_oracle.cpp) thresholded strictly and above 1e-8, with seeds at the pixels
not below any 3 x 3 neighbour (Segmentation2D.cpp:294-333, the frame surrounded by zeros). The shapes cover one strip,
ragged last strips and row blocks, unaligned and aligned widths (the vector-load path), frames 16 rows high and
several frames; threshold 0 makes most pixels domain, so the per-warp list stages fill and move many times.
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
    src = src.replace('#include "async_copy.cuh"', '#include "async_copy_emu.h"')  # copies at once, checks alignment
    # dynamic shared memory: a static buffer (blocks run one at a time)
    return re.sub(r'extern __shared__ (__align__\(\d+\) )?([\w ]+?) (\w+)\[\];', r'static \1\2 \3[262144];', src)


@pytest.fixture(scope="module")
def emulators(tmp_path_factory):
    if shutil.which("g++") is None or not os.path.exists(os.path.join(CUDA_INCLUDE, "cuda_runtime.h")):
        pytest.skip("g++ or the CUDA headers are missing")
    exes = {}
    for name, fname, cuts, flag in (
            ("tiles", "detect.cu", [("bool ConfigureSmem()", "}  // namespace\n"),
                                    ("long long ThresholdFixed(", "}  // namespace ptb")], None),
            ("stream", "detect_stream.cu", [("template <bool kVec> bool LaunchStream(", "}  // namespace\n"),
                                            ("bool StreamDetectFits(", "}  // namespace ptb")], "-DPTB_EMU_STREAM")):
        d = tmp_path_factory.mktemp("emu_" + name)
        open(d / "detect_emu.inc", "w").write(_kernels_only(open(os.path.join(CSRC, fname)).read(), cuts))
        exe = d / "emu_detect"
        cmd = ["g++", "-std=c++20", "-O2", "-g", "-fsanitize=address", "-pthread", "-Wno-attributes",
               "-I" + CUDA_INCLUDE, "-I" + str(d), "-I" + os.path.join(HERE, "emu")]
        cmd += [flag] if flag else []
        cmd += [os.path.join(HERE, "emu", "detect_driver.cpp"), "-o", str(exe)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-3000:]
        exes[name] = exe
    return exes


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


CASES = [  # (H, W, frames, seed)
    (130, 112, 2, 1),   # exactly one strip, two row blocks (the second of 2 rows)
    (300, 250, 1, 2),   # three strips, the last of 26 columns; odd width: scalar loads
    (140, 232, 2, 3),   # width a multiple of 4: the middle strip takes the vector loads
    (16, 336, 1, 4),    # 16 rows, three full strips
    (129, 225, 1, 5),   # last strip of one column
    (270, 116, 1, 6),   # vector loads, a last strip of 4 columns, two row blocks (the second of 14 rows)
    (257, 113, 1, 7),   # a last row block of one row, a last strip of one column
]


@pytest.mark.parametrize("case", CASES, ids=["x".join(map(str, c[:3])) for c in CASES])
def test_stream_detection_matches_tiles_and_oracle(emulators, orc, case):
    import synth
    h, w, b, seed = case
    stack, _ = synth.stack("c2", frames=b, seed=seed, size=(h, w))
    base = synth.mad_threshold(orc.planes(stack[0])[1])
    for thr in (int(np.floor(base * 65536)), int(np.floor(0.3 * base * 65536)), 0, -5):
        want_code, want_w1 = _expected(orc, stack, thr)
        got = {k: _run(exe, stack, thr) for k, exe in emulators.items()}
        for name, g in got.items():
            assert g["overflow"] == 0, name
            assert np.array_equal(g["code"], want_code), (name, thr, int(np.sum(g["code"] != want_code)))
            assert np.array_equal(g["w1"], want_w1), (name, thr)
            dom_idx = np.flatnonzero(want_code & 1).astype(np.uint32)
            seed_idx = np.flatnonzero(want_code & 2).astype(np.uint32)
            assert np.array_equal(g["dom"], dom_idx), name
            assert np.array_equal(g["seeds"], seed_idx), name
            per = (want_code.reshape(b, -1) & 1).sum(axis=1)
            assert np.array_equal(g["fdom"], per), name
            assert np.array_equal(g["fseed"], ((want_code.reshape(b, -1) & 2) != 0).sum(axis=1)), name
