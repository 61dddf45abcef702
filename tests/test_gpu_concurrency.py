"""Concurrent calls of the C ABI from several host threads (the reference is reentrant, CPU/main.cpp:18-26).

Each call leases its own engine of the device's pool, so four threads calling Localization and Fitting at once must
get exactly the rows of the same calls made one after the other, while running side by side on the GPU.
"""
import threading
import time

import numpy as np
import pytest

from conftest import GAUSS_PARAMS

pytestmark = pytest.mark.gpu

MLE6 = np.array([7.0, 1.3, 100.0, 2.0, 20.0, 0.0])


def _positions(rows):
    return np.ascontiguousarray(np.stack([rows[:, 0], rows[:, 1], rows[:, 4], rows[:, 5], rows[:, 15], rows[:, 16]], axis=1))


def _work(lib, stack, thr):
    a = lib.localization(stack, thr, 0.0, 6, MLE6)
    b = lib.fitting(stack, _positions(a), 2, GAUSS_PARAMS)
    c = lib.localization(stack, thr, 10.0, 0, GAUSS_PARAMS)
    return a, b, c


def test_four_threads_match_serial_calls(lib, orc, monkeypatch):
    import synth
    # one ROI mapping for every engine (each engine autotunes on its own; the mapping changes the last FP32 bits)
    monkeypatch.setenv("PTB_MLE_LANES", "1")
    stacks = [synth.stack("c1", frames=24, seed=300 + i)[0] for i in range(4)]
    thrs = [synth.mad_threshold(orc.planes(s[0])[1]) for s in stacks]
    for s, t in zip(stacks, thrs):
        _work(lib, s, t)  # warm-up: kernels loaded, first engine sized
    t0 = time.perf_counter()
    serial = [_work(lib, s, t) for s, t in zip(stacks, thrs)]
    serial_s = time.perf_counter() - t0

    results = [None] * 4
    errors = []
    start = threading.Barrier(4)

    def run(i):
        try:
            start.wait()
            results[i] = _work(lib, stacks[i], thrs[i])
        except Exception as ex:  # reported below: a thread's failure must fail the test
            errors.append(ex)

    for rep in range(2):  # the second round reuses the engines the first one created
        threads = [threading.Thread(target=run, args=(i,)) for i in range(4)]
        t0 = time.perf_counter()
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        concurrent_s = time.perf_counter() - t0
        assert not errors, errors
        for got, want in zip(results, serial):
            for g, w in zip(got, want):
                assert g.shape == w.shape and np.array_equal(g, w)
    stats = lib.engine_pool_stats()
    print("serial %.1f ms, four threads %.1f ms, pool %s" % (serial_s * 1e3, concurrent_s * 1e3, stats))
    assert stats["engines"] >= 2 and stats["peak_leased"] >= 2


def test_settings_apply_to_every_engine(lib, orc):
    """A setting changed through the C ABI holds for the engines the pool creates later too."""
    import synth
    s, _ = synth.stack("c2", frames=2, seed=21, size=(256, 256))
    thr = 0.1 * synth.mad_threshold(orc.planes(s[0])[1])
    prev = lib.set_segmentation_mode(1)
    try:
        out = [None] * 3

        def run(i):
            lib.segmentation_stats()
            out[i] = lib.localization(s, thr, 0.0, 0, GAUSS_PARAMS)

        threads = [threading.Thread(target=run, args=(i,)) for i in range(3)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        want = orc.localization(s, thr, 0.0, 0, GAUSS_PARAMS)
        for o in out:
            assert np.array_equal(o, want)
        # strict mode floods every frame as one unit: nothing is counted as routed
        assert lib.segmentation_stats()["routed"] == 0
    finally:
        lib.set_segmentation_mode(prev)
