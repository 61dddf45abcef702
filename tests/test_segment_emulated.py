"""The segmentation kernels run on the CPU under AddressSanitizer, against the oracle's labels.

tests/emu/shim.h runs every CUDA thread of a block as a host thread (blocks one after another, warp shuffles and
ballots on per-warp barriers, __syncthreads on a block barrier) and tests/emu/driver.cpp drives the kernels of
palmtracer-cpp_b200/csrc/segment.cu in the engine's launch order on one frame, each device array its own heap
allocation: an out-of-bounds access anywhere in them aborts under AddressSanitizer, and the labels must equal the
oracle's (Segmentation2D.cpp:336-385 restated in oracle/pt_oracle.cpp). The frames exercise the first exactness test,
the rank test, the re-flood with estimated frame-wide aging (in shared-memory boxes and, for groups larger than a box,
in global memory) and the frame-wide flood.
"""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CUDA_INCLUDE = "/usr/local/cuda/include"


@pytest.fixture(scope="module")
def emulator(tmp_path_factory):
    if shutil.which("g++") is None or not os.path.exists(os.path.join(CUDA_INCLUDE, "cuda_runtime.h")):
        pytest.skip("g++ or the CUDA headers are missing")
    d = tmp_path_factory.mktemp("emu")
    src = open(os.path.join(ROOT, "palmtracer-cpp_b200", "csrc", "segment.cu")).read()
    # the kernels and device functions only: the host launch function uses the <<< >>> syntax
    cut = src.index("bool LaunchSegment(")
    end = src.rindex("}  // namespace ptb")
    src = src[:cut] + src[end:]
    common = os.path.join(ROOT, "palmtracer-cpp_b200", "csrc", "pt_common.cuh")
    src = re.sub(r'#include "pt_common.cuh"', '#include "%s"' % common, src)
    # dynamic shared memory: a static buffer (blocks run one at a time)
    src = re.sub(r'extern __shared__ (\w+) (\w+)\[\];', r'static \1 \2[65536];', src)
    open(d / "segment_emu.inc", "w").write(src)
    exe = d / "emu"
    cmd = ["g++", "-std=c++20", "-O2", "-g", "-fsanitize=address", "-pthread", "-Wno-attributes", "-I" + CUDA_INCLUDE,
           "-I" + str(d), "-I" + os.path.join(HERE, "emu"), os.path.join(HERE, "emu", "driver.cpp"), "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return exe, d


def _run(emulator, orc, frame, thr, mode=0):
    exe, d = emulator
    h, w = frame.shape
    w1 = orc.planes(frame)[1]
    fixed = np.round(w1 * 65536).astype(np.int64)
    assert np.array_equal(fixed, w1 * 65536)  # W1 is an exact multiple of 2^-16
    inp, out = d / "in.bin", d / "out.bin"
    with open(inp, "wb") as f:
        np.array([h, w], dtype=np.int32).tofile(f)
        np.array([int(np.floor(thr * 65536))], dtype=np.int64).tofile(f)
        fixed.tofile(f)
    r = subprocess.run([str(exe), str(inp), str(out), str(mode)], capture_output=True, text=True,
                       env=dict(os.environ, ASAN_OPTIONS="detect_leaks=0"), timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    raw = np.fromfile(out, dtype=np.uint8)
    n = h * w
    lab = raw[:4 * n].view(np.uint32)
    code = raw[4 * n:5 * n]
    stats = dict(zip(("routed", "rank_tested", "reflooded", "pairs", "fits", "global_reflood_groups"),
                     map(int, raw[5 * n:].view(np.uint32))))
    dom = (code & 1) != 0
    want = orc.labels(frame, thr, 0.0).reshape(-1)
    return int(np.sum(lab[dom] != want[dom])), stats


def test_emulated_segmentation_matches_oracle(emulator, orc):
    import synth
    s, _ = synth.stack("c2", frames=1, seed=21, size=(512, 512))
    base = synth.mad_threshold(orc.planes(s[0])[1])
    seen = {"rank_tested": 0, "reflooded": 0, "routed": 0, "global_reflood_groups": 0}
    for scale, mode in ((1.0, 0), (0.5, 0), (0.3, 0), (0.15, 0), (0.3, 2)):
        diff, stats = _run(emulator, orc, s[0], base * scale, mode)
        print("scale", scale, "mode", mode, stats, "label differences", diff)
        assert diff == 0, (scale, mode, stats)
        for k in seen:
            seen[k] += stats[k]
    assert all(v >= 1 for v in seen.values()), seen


def test_emulated_segmentation_noise_frame(emulator, orc):
    """Full-range noise at and just above threshold 0: about half the pixels join the domain in components of
    arbitrary shape, so many pixels join two union-find trees (the union pass's list), the chains walked by the
    component count are long, and most frames' groups are large."""
    rng = np.random.default_rng(5)
    frame = rng.integers(0, 65536, size=(150, 230), dtype=np.uint16)
    w1 = orc.planes(frame)[1]
    for thr in (0.0, float(np.quantile(w1[w1 > 0], 0.5))):
        diff, stats = _run(emulator, orc, frame, thr, 0)
        print("thr", thr, stats, "label differences", diff)
        assert diff == 0, (thr, stats)
